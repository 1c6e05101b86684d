"""Extract the Farrell (1972) elastic load Green's function table that the reference
ships as src/input/elasticgreencoeffs_farrell1972.jld2 (the table its
get_greenintegrand_coeffs downloads at run time, src/dataloaders.jl:257-273).

The JLD2 file holds three little-endian float64[42] arrays at fixed byte offsets:
angle (deg) at 622, distance rm (m) at 1024 and the coefficients GE at 1426.  This
script reads those bytes from a FastIsostasy.jl checkout and writes
elasticgreencoeffs_farrell1972.txt (columns: angle, rm, GE) next to itself.

usage: python make_farrell_table.py <path-to-FastIsostasy.jl>
"""
import pathlib
import struct
import sys

OFFSETS = {"angle": 622, "rm": 1024, "GE": 1426}
N = 42


def main(repo: str) -> None:
    blob = (pathlib.Path(repo) / "src" / "input" / "elasticgreencoeffs_farrell1972.jld2").read_bytes()
    cols = {k: struct.unpack("<%dd" % N, blob[o:o + 8 * N]) for k, o in OFFSETS.items()}
    assert cols["rm"][0] == 0.0 and all(b > a for a, b in zip(cols["rm"], cols["rm"][1:]))
    out = pathlib.Path(__file__).resolve().parent / "elasticgreencoeffs_farrell1972.txt"
    with open(out, "w") as f:
        f.write("# angle_deg distance_m GE  (Farrell 1972, table A3; extracted by make_farrell_table.py)\n")
        for a, r, g in zip(cols["angle"], cols["rm"], cols["GE"]):
            f.write(f"{a!r} {r!r} {g!r}\n")
    print(f"wrote {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
