"""Ensemble sharding over GPUs (one process per GPU, torch.distributed for plumbing).

Members are independent, so an ensemble splits across ranks with no communication in
the time loop: each rank steps its own share with the persistent ensemble executor and
the ranks meet once at the end to gather statuses and timings.  Shares are balanced by
greedy bin-packing on a member's expected cost over a window: the cost of one step
attempt, about N^2 log2 N, times the number of attempts, which scales with the member's
stiffest relaxation rate (`stiffness_rate`): the adaptive BS3 step stays inside the
method's stability region, so its attempts per simulated year grow with that rate.
"""
from __future__ import annotations

import math

SECONDS_PER_YEAR = 60.0**2 * 24 * 365.25


def stiffness_rate(eta_min, D, dx, dy=None, rho_m=3.4e3, g=9.8):
    """The fastest viscous relaxation rate of a member (1/yr): the rate
    (D |k|^4 + rho_m g) / (2 eta |k|) of the LV-ELVA operator (src/deformation.jl:91-131
    linearised about a uniform Earth) at the grid's largest wavenumber and the member's
    smallest effective viscosity."""
    dy = dx if dy is None else dy
    k = math.pi * math.sqrt(1.0 / dx**2 + 1.0 / dy**2)
    return (D * k**4 + rho_m * g) / (2.0 * eta_min * k) * SECONDS_PER_YEAR


def member_cost(n, rate=1.0):
    """Expected cost over a window: N^2 log2 N per attempt times the attempt rate."""
    return float(n) * float(n) * math.log2(max(float(n), 2.0)) * float(rate)


def shard_members(sizes, world, rates=None):
    """Partition member indices over `world` ranks: costliest first onto the lightest
    rank (ties by rank).  rates: each member's stiffness_rate (None: all equal).
    Every rank computes the same answer.  Returns one ascending index list per rank."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    rates = [1.0] * len(sizes) if rates is None else list(rates)
    cost = [member_cost(n, r) for n, r in zip(sizes, rates)]
    order = sorted(range(len(sizes)), key=lambda i: (-cost[i], i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += cost[i]
    return [sorted(p) for p in parts]


def member_rate(member, litho_thickness=100e3, E=6.6e10, nu=0.28):
    """stiffness_rate of a config-3 style member dict (log10eta map, domain), with the
    effective viscosity of a compressible mantle (x 1.5 / (1 + nu_m), src/material.jl:46-52)
    and the rigidity of its lithosphere (src/material.jl:10)."""
    D = E * litho_thickness**3 / (12.0 * (1.0 - nu**2))
    eta_min = 10.0 ** float(min(map(float, member["log10eta"].ravel()))) * 1.5 / 1.28
    d = member["domain"]
    return stiffness_rate(eta_min, D, d.dx, d.dy)


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

    mine = shard_members([m["N"] for m in members], world, [member_rate(m) for m in members])[rank]
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
