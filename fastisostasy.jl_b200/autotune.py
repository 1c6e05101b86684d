"""Tile and FFT-schedule autotuner of the FP32 kernels (no counterpart in the reference).

The FP32 form's row phases work on tiles of ``h`` rows (row FFTs, stencils with a
two-row halo) and its column phase on blocks of ``B`` spectral columns.  Small tiles
give a single simulation the most parallelism (it is latency-bound); tall tiles cut
the halo recomputation and suit an ensemble (throughput-bound).  This module measures
candidate (h, B) pairs on the actual workload with the library's own device timers and
records the fastest per workload key in a JSON table shipped with the package
(``tuning/b200.json``); ``tiles_for`` reads it back.

The transforms (row and column FFTs of length N, padded convolutions of length M) run
Stockham passes in a radix order; ``fft`` measures candidate orders of each length's
factors (radices 2, 3, 4, 5, 7, 8) per BS3 step of the single-simulation workload
at that N and records the fastest as "fft:<L>"; ``fft_schedule_for`` reads it back and
``Simulation`` applies it through fi_set_fft_schedule.

    python fastisostasy.jl_b200/autotune.py single 350     # config-2 grid (persistent executor)
    python fastisostasy.jl_b200/autotune.py ensemble 128   # config-3 ensemble
    python fastisostasy.jl_b200/autotune.py fft 350        # radix order of the length-350 transforms
    python fastisostasy.jl_b200/autotune.py ensemble-rule 128   # per-member tiles h = B = c / N

Ensemble members of different N get different tiles under the per-member rule, so that a
task (tile of one member) costs about the same whatever the member's grid.
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


def ensemble_rule_for():
    """The tuned per-member tile rule of ensembles, c: member of grid N gets h = B =
    clamp(c // N, 2, 16) (tasks of similar size across members), or None."""
    if os.environ.get("FI_NO_TUNING") == "1":
        return None
    v = _load().get("ensemble:per_n")
    return int(v["c"]) if v else None


def rule_tiles(c, N):
    t = max(2, min(16, int(c) // int(N)))
    return (t, t)


def time_ensemble_rule(n_members, c, years=1000.0, warm=50.0):
    """Device ms per simulated member-year of the config-3 ensemble with per-member tiles
    h = B = clamp(c // N, 2, 16)."""
    members, t_ice, mod = W.config3_members(n_members=n_members)
    sims = [W.config3_simulation(m, t_ice, mod, form="fp32") for m in members]
    for s, m in zip(sims, members):
        s.cfg.max_steps = 50_000_000
        s.tiles = rule_tiles(c, m["N"])
    ens = M.Ensemble(sims, tiles=None)
    ens.step(warm)
    ens.step(years)
    ms = ens.last_gpu_ms / (years * n_members)
    ens.close()
    for s in sims:
        s.close()
    return ms


def tune_ensemble_rule(n_members=128, candidates=(1024, 1536, 2048, 2560, 3072, 4096), write=True):
    results = {}
    for c in candidates:
        results[c] = time_ensemble_rule(n_members, c)
        print(json.dumps({"kind": "ensemble rule", "c": c, "ms_per_member_year": results[c]}), flush=True)
    best = min(results, key=results.get)
    entry = {"c": best, "ms_per_unit": results[best], "unit": "ms per simulated member-year (config 3, 1 kyr)",
             "rule": "h = B = clamp(c // N, 2, 16)", "candidates": {str(k): v for k, v in results.items()}}
    if write:
        table = _load()
        table["ensemble:per_n"] = entry
        TABLE_DIR.mkdir(exist_ok=True)
        TABLE.write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
    return "ensemble:per_n", entry


def fft_schedule_for(L):
    """The tuned radix order for transforms of length L, or None (FI_NO_TUNING=1 or
    FI_NO_FFT_TUNING=1: the library's default order)."""
    if os.environ.get("FI_NO_TUNING") == "1" or os.environ.get("FI_NO_FFT_TUNING") == "1":
        return None
    v = _load().get(f"fft:{L}")
    return list(v["schedule"]) if v else None


REG_RADICES = (8, 7, 5, 4, 3, 2)


def default_schedule(L):
    """The library's default order (fi_api.cu: radix 8 while possible, then 4, 2, 7, 5,
    3, larger odd factors)."""
    m, out = L, []
    for r in (8, 4, 2, 7, 5, 3):
        while m % r == 0:
            out.append(r)
            m //= r
    f = 11
    while f * f <= m:
        while m % f == 0:
            out.append(f)
            m //= f
        f += 2
    if m > 1:
        out.append(m)
    return out


def schedule_candidates(L, limit=12, max_passes=6):
    """Radix orders for length L: the library default, then the orderings of the
    factorisations of L into register radices with the fewest passes first (at most
    `limit` in all)."""
    out = set()

    def grow(m, acc):
        if len(acc) > max_passes:
            return
        if m == 1:
            out.add(tuple(acc))
            return
        for r in REG_RADICES:
            if m % r == 0:
                grow(m // r, acc + [r])

    grow(L, [])
    dflt = default_schedule(L)
    cands = [c for c in sorted(out, key=lambda t: (len(t), t)) if list(c) != dflt]
    return [dflt] + [list(c) for c in cands[:limit - 1]]


def time_single_per_step(N, tiles=None, schedules=None, years=5.0, warm=5.0):
    """Device ms per BS3 attempt of the config-2 workload at grid N (independent of the
    step count, which the rounding of different schedules may change by a few steps)."""
    sim = W.config2(form="fp32", N=N)
    sim.tiles = tiles
    sim.fft_schedules = dict(schedules or {})
    sim.cfg.max_steps = 50_000_000
    integ = M.init_integrator(sim)
    M.step(integ, warm, True)
    a0 = sim.stats()
    M.step(integ, years, True)
    a1 = sim.stats()
    att = (a1["naccept"] + a1["nreject"]) - (a0["naccept"] + a0["nreject"])
    sim.close()
    return a1["last_gpu_ms"] / max(1, att)


def tune_fft(N, write=True, limit=12):
    """Radix orders of the length-N transforms (rows and columns of an N x N grid)."""
    results = {}
    for c in schedule_candidates(N, limit=limit):
        try:
            results[tuple(c)] = time_single_per_step(N, schedules={N: c})
        except Exception as ex:
            results[tuple(c)] = float("inf")
            print(f"schedule {c}: {ex}", file=sys.stderr)
        print(json.dumps({"kind": "fft", "L": N, "schedule": c, "ms_per_bs3_step": results[tuple(c)]}), flush=True)
    best = min(results, key=results.get)
    key = f"fft:{N}"
    entry = {"schedule": list(best), "ms_per_unit": results[best], "unit": "ms per BS3 step (config-2 workload)",
             "candidates": {"x".join(map(str, k)): v for k, v in results.items()}}
    if write:
        table = _load()
        table[key] = entry
        TABLE_DIR.mkdir(exist_ok=True)
        TABLE.write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
    return key, entry


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
    size = int(sys.argv[2]) if len(sys.argv) > 2 else (128 if kind == "ensemble" else 350)
    if kind == "fft":
        res = tune_fft(size)
    elif kind == "ensemble-rule":
        res = tune_ensemble_rule(size)
    else:
        res = tune(kind, size)
    print(json.dumps(dict(zip(("key", "entry"), res))))
