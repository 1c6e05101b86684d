"""Tile autotuner of the FP32 kernels (no counterpart in the reference).

The FP32 form's row phases work on tiles of ``h`` rows (row FFTs, stencils with a
two-row halo) and its column phase on blocks of ``B`` spectral columns.  Small tiles
give a single simulation the most parallelism (it is latency-bound); tall tiles cut
the halo recomputation and suit an ensemble (throughput-bound).  This module measures
candidate (h, B) pairs on the actual workload with the library's own device timers and
records the fastest per workload key in a JSON table shipped with the package
(``tuning/b200.json``); ``tiles_for`` reads it back.

    python fastisostasy.jl_b200/autotune.py single 350     # config-2 grid (persistent executor)
    python fastisostasy.jl_b200/autotune.py ensemble 128   # config-3 ensemble
"""
from __future__ import annotations

import json
import os
import pathlib
import sys

if __package__ in (None, ""):  # run as a script: load the package by its import name
    sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1]))
    import __graft_entry__  # noqa: E402

    __graft_entry__.load_package()
    from fastiso_b200 import model as M  # noqa: E402
    from fastiso_b200 import workloads as W  # noqa: E402
else:
    from . import model as M
    from . import workloads as W

TABLE_DIR = pathlib.Path(__file__).resolve().parent / "tuning"
TABLE = TABLE_DIR / "b200.json"

SINGLE_CANDIDATES = [(1, 1), (1, 2), (2, 1), (2, 2), (2, 4), (3, 2), (4, 4)]
ENSEMBLE_CANDIDATES = [(2, 2), (4, 4), (8, 4), (8, 8), (12, 8), (16, 8), (16, 16)]


def _load():
    try:
        return json.loads(TABLE.read_text())
    except Exception:
        return {}


def tiles_for(key):
    """The tuned (h, B) for a workload key such as "single:350" or "ensemble:128"."""
    if os.environ.get("FI_NO_TUNING") == "1":
        return None
    v = _load().get(key)
    return tuple(v["tiles"]) if v else None


def time_single(N, tiles, years=20.0, warm=10.0):
    """Device ms per simulated year of the config-2 workload at grid N with these tiles."""
    sim = W.config2(form="fp32", N=N)
    sim.tiles = tiles
    sim.cfg.max_steps = 50_000_000
    integ = M.init_integrator(sim)
    M.step(integ, warm, True)
    M.step(integ, years, True)
    ms = sim.stats()["last_gpu_ms"] / years
    sim.close()
    return ms


def time_ensemble(n_members, tiles, years=300.0, warm=50.0):
    """Device ms per simulated member-year of the config-3 ensemble with these tiles."""
    members, t_ice, mod = W.config3_members(n_members=n_members)
    sims = [W.config3_simulation(m, t_ice, mod, form="fp32") for m in members]
    for s in sims:
        s.cfg.max_steps = 50_000_000
    ens = M.Ensemble(sims, tiles=tiles)
    ens.step(warm)
    ens.step(years)
    ms = ens.last_gpu_ms / (years * n_members)
    ens.close()
    for s in sims:
        s.close()
    return ms


def tune(kind, size, candidates=None, write=True):
    cands = candidates or (SINGLE_CANDIDATES if kind == "single" else ENSEMBLE_CANDIDATES)
    results = {}
    for c in cands:
        try:
            results[c] = time_single(size, c) if kind == "single" else time_ensemble(size, c)
        except Exception as ex:  # a candidate that does not fit the shared-memory budget
            results[c] = float("inf")
            print(f"candidate {c}: {ex}", file=sys.stderr)
        print(json.dumps({"kind": kind, "size": size, "tiles": list(c), "ms_per_unit": results[c]}), flush=True)
    best = min(results, key=results.get)
    key = f"{kind}:{size}"
    entry = {"tiles": list(best), "ms_per_unit": results[best],
             "unit": "ms per simulated year" if kind == "single" else "ms per simulated member-year",
             "candidates": {f"{h}x{b}": v for (h, b), v in results.items()}}
    if write:
        table = _load()
        table[key] = entry
        TABLE_DIR.mkdir(exist_ok=True)
        TABLE.write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
    return key, entry


if __name__ == "__main__":
    kind = sys.argv[1] if len(sys.argv) > 1 else "single"
    size = int(sys.argv[2]) if len(sys.argv) > 2 else (350 if kind == "single" else 128)
    print(json.dumps(dict(zip(("key", "entry"), tune(kind, size)))))
