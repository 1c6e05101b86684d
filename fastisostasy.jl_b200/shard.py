"""Ensemble sharding over GPUs (one process per GPU, torch.distributed for plumbing).

Members are independent, so an ensemble splits across ranks with no communication in
the time loop: each rank steps its own share with the persistent ensemble executor and
the ranks meet once at the end to gather statuses and timings.  Shares are balanced by
greedy bin-packing on the cost of a step, about N^2 log2 N per member (a member's step
count is not known in advance).
"""
from __future__ import annotations

import math


def member_cost(n):
    return float(n) * float(n) * math.log2(max(float(n), 2.0))


def shard_members(sizes, world):
    """Partition member indices over `world` ranks: largest first onto the lightest rank
    (ties by rank).  Every rank computes the same answer.  Returns one ascending index
    list per rank."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-member_cost(sizes[i]), i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += member_cost(sizes[i])
    return [sorted(p) for p in parts]


def gather_results(local, world):
    """All ranks' result dicts, in rank order (one all_gather_object at the end of a run)."""
    if world == 1:
        return [local]
    import torch.distributed as dist

    out = [None] * world
    dist.all_gather_object(out, local)
    return out


def run_shard(members, t_ice, mod, years, rank, world, device=0, warm=50.0):
    """Steps this rank's share of a config-3 style ensemble; returns the gathered
    per-rank results (member indices, statuses, device ms)."""
    from . import model as M
    from . import workloads as W

    mine = shard_members([m["N"] for m in members], world)[rank]
    res = {"rank": rank, "members": mine, "status": [], "ms": 0.0, "attempts": []}
    if mine:
        sims = [W.config3_simulation(members[i], t_ice, mod, form="fp32") for i in mine]
        for s in sims:
            s.cfg.device = device
            s.cfg.max_steps = 50_000_000
        ens = M.Ensemble(sims)
        ens.step(warm)
        a0 = [s.stats() for s in sims]
        res["status"] = ens.step(years)
        res["ms"] = ens.last_gpu_ms
        a1 = [s.stats() for s in sims]
        # step attempts of each member in the timed window
        res["attempts"] = [(b["naccept"] + b["nreject"]) - (a["naccept"] + a["nreject"]) for a, b in zip(a0, a1)]
        ens.close()
        for s in sims:
            s.close()
    return gather_results(res, world)
