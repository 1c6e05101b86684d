"""Surrogate of a 100-yr macro-step of the LV-ELVA solver, and the screening loop in which
the plain solver checks its proposals.  No counterpart in FastIsostasy.jl (its closest
precedent is the threaded ensemble of ext/FastIsostasyEnsembleKalmanProcessesExt.jl:107-122,
which runs the solver for every candidate).

Pipeline
  1. ``member_spec`` draws a config-1-style member on an S x S grid from a seed: a
     log10-viscosity random field, a lithosphere-thickness random field and an ice sheet
     (parabolic dome of random centre, radius and height) switched on over the first year.
  2. ``generate_trajectories`` runs the members with the GPU solver (the persistent
     ensemble kernel, FP32 form) and records u every 100 yr.
  3. ``Dataset`` keeps the trajectories on the GPU; a sample is
     x = (u/100 m, H/1000 m, (log10 eta - 21)/0.5, (T - 100 km)/25 km, x, y) at t and the
     target (u(t + 100 yr) - u(t)) / 10 m.
  4. ``train`` runs the FNO's own CUDA forward, backward and Adam (``fno.FNO``).
  5. ``rollout`` chains macro-steps; ``evaluate`` reports rel-L2 per macro-step and after
     the full rollout on held-out members.
  6. ``screen``: the surrogate rolls every candidate of a pool forward and proposes them in
     order of predicted misfit to an observation; the plain solver runs each proposal,
     accepts it when its own result fits the observation and the surrogate's prediction
     was within ``bound`` of it, and otherwise replaces it by the next proposal.  Accepted
     members therefore carry the solver's states.  ``screen_without_surrogate`` is the
     same loop on the solver alone (candidates in random order).

Array layout: every grid array here is [j, i] (x fastest), the network's layout; the
solver's (nx, ny) arrays are transposed on the way in.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import model as M
from .workloads import gaussian_random_field

MACRO_DT = 100.0
U_SCALE, DU_SCALE, H_SCALE = 100.0, 10.0, 1000.0
ETA_MEAN, ETA_SCALE = 21.0, 0.5
T_MEAN, T_SCALE = 100e3, 25e3


@dataclass
class MemberSpec:
    seed: int
    N: int
    W: float
    log10eta: np.ndarray   # (nx, ny), solver layout
    T: np.ndarray          # lithosphere thickness (m)
    H: np.ndarray          # ice thickness (m) after the first year
    meta: dict = field(default_factory=dict)


def member_spec(seed, N=128, W=1.5e6, eta_mean=None, ice=None, T=None, eta_pattern=None, eta_amp=0.5):
    """A config-1-style member drawn from `seed`: log10 eta = mean + eta_amp g (g a unit
    Gaussian random field, l = 500 km, unless eta_pattern is given; mean ~ U[20, 22]
    unless eta_mean is given), T and the ice dome random unless given (a candidate pool
    shares them)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    domain = M.RegionalDomain(W, W, N, N)
    mean = rng.uniform(20.0, 22.0) if eta_mean is None else float(eta_mean)
    g = gaussian_random_field(N, N, W, W, 500e3, 7000 + seed) if eta_pattern is None else eta_pattern
    log10eta = np.clip(mean + eta_amp * g, 19.0, 23.0)
    if T is None:
        gT = gaussian_random_field(N, N, W, W, 500e3, 17000 + seed)
        T = np.clip(100e3 + 25e3 * gT, 50e3, 170e3)
    if ice is None:
        cx, cy = rng.uniform(-0.3 * W, 0.3 * W, 2)
        R = rng.uniform(0.25 * W, 0.6 * W)
        H0 = rng.uniform(500.0, 2500.0)
        r2 = ((domain.X - cx) ** 2 + (domain.Y - cy) ** 2) / R**2
        ice = H0 * np.sqrt(np.clip(1.0 - r2, 0.0, None))
    return MemberSpec(seed, N, W, log10eta, np.asarray(T, float), np.asarray(ice, float),
                      {"eta_mean": mean, "eta_amp": eta_amp, "eta_pattern": g})


def simulation_for(spec: MemberSpec, t_end: float):
    domain = M.RegionalDomain(spec.W, spec.W, spec.N, spec.N)
    N = spec.N
    se = M.SolidEarth(domain, layer_boundaries=spec.T.reshape(N, N, 1),
                      layer_viscosities=(10.0 ** spec.log10eta).reshape(N, N, 1))
    it = M.TimeInterpolatedIceThickness([0.0, 1.0, t_end + MACRO_DT], [domain.zeros(), spec.H, spec.H], domain)
    bcs = M.BoundaryConditions(domain, ice_thickness=it)
    return M.Simulation(domain, bcs, M.RegionalSeaLevel(), se, (0.0, t_end + MACRO_DT),
                        nout=M.NativeOutput(t=[t_end]), form="fp32")


def generate_trajectories(specs, t_end=10e3, batch=128, every=MACRO_DT, log=None, device=None):
    """u every `every` years from 0 to t_end for each member: float32 [n, K + 1, N, N]
    ([j, i] layout), a numpy array or, with `device`, a torch tensor there.  Members
    advance together in the persistent ensemble kernel, batched in order of mean
    viscosity so that a batch's members need similar step counts."""
    K = int(round(t_end / every))
    N = specs[0].N
    order = np.argsort([float(np.mean(s.log10eta)) for s in specs], kind="stable")
    if device is None:
        out = np.zeros((len(specs), K + 1, N, N), dtype=np.float32)
    else:
        import torch

        out = torch.zeros((len(specs), K + 1, N, N), dtype=torch.float32, device=device)
    for b0 in range(0, len(specs), batch):
        idx = order[b0:b0 + batch]
        part = [specs[i] for i in idx]
        sims = [simulation_for(s, t_end) for s in part]
        ens = M.Ensemble(sims)
        for k in range(1, K + 1):
            st = ens.step(every)
            if any(st):
                bad = [part[i].seed for i, s in enumerate(st) if s]
                raise RuntimeError(f"solver failed for members {bad}: status {st}")
            snap = np.stack([sim.get_field("u").T for sim in sims]).astype(np.float32)
            if device is None:
                out[idx, k] = snap
            else:
                out[torch.as_tensor(idx, device=device), k] = torch.from_numpy(snap).to(device)
        ens.close()
        for s in sims:
            s.close()
        if log:
            log(f"trajectories {b0 + len(part)}/{len(specs)}")
    return out


def static_features(spec: MemberSpec):
    """(H, log10 eta, T, x, y) normalised, float32 [5, N, N] in [j, i] layout."""
    N = spec.N
    c = np.linspace(-1.0, 1.0, N, dtype=np.float64)
    X, Y = np.meshgrid(c, c, indexing="ij")
    f = np.stack([spec.H / H_SCALE, (spec.log10eta - ETA_MEAN) / ETA_SCALE, (spec.T - T_MEAN) / T_SCALE, X, Y])
    return np.ascontiguousarray(f.transpose(0, 2, 1)).astype(np.float32)


class Dataset:
    """Trajectories and static features resident on the GPU."""

    def __init__(self, specs, u, device="cuda"):
        import torch

        self.specs = list(specs)
        if isinstance(u, torch.Tensor):
            self.u = u.to(device).contiguous()                                           # [n, K+1, N, N]
        else:
            self.u = torch.from_numpy(np.ascontiguousarray(u)).to(device)
        self.static = torch.from_numpy(np.stack([static_features(s) for s in specs])).to(device)  # [n, 5, N, N]
        self.n, self.K = self.u.shape[0], self.u.shape[1] - 1
        self.N = self.u.shape[-1]
        # loss weight of each trajectory: 1 / mean-square displacement at the end (so that
        # every member's rollout counts relative to its own size), normalised to mean 1
        ms = (self.u[:, -1] ** 2).mean(dim=(-2, -1)).clamp_min(1.0)
        self.w = (1.0 / ms) / (1.0 / ms).mean()

    def inputs(self, traj, k):
        import torch

        u = self.u[traj, k]
        return torch.cat([(u / U_SCALE).unsqueeze(1), self.static[traj]], dim=1).contiguous()

    def batch(self, traj, k):
        x = self.inputs(traj, k)
        y = ((self.u[traj, k + 1] - self.u[traj, k]) / DU_SCALE).contiguous()
        return x, y


def dp_step(net, x, y, w, lr, group=None):
    """One training step, data-parallel when torch.distributed runs more than one rank:
    the local forward, loss and backward (``net.loss_backward``), the gradient vector
    averaged over the ranks in place (one all-reduce of num_params floats; NCCL over
    NVLink on GPUs), then Adam on every rank.  Ranks that start from the same parameters
    stay identical.  Returns the loss averaged over the ranks."""
    import torch
    import torch.distributed as dist

    loss = net.loss_backward(x, y, w)
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if world > 1:
        g = net.grads_tensor()
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
        g /= world
        lt = torch.tensor([loss], dtype=torch.float32, device=g.device)
        dist.all_reduce(lt, op=dist.ReduceOp.SUM, group=group)
        loss = float(lt.item()) / world
        if g.is_cuda:
            torch.cuda.synchronize(g.device)  # the averaged gradients are in place before Adam
    net.adam(lr)
    return loss


def train(net, data: Dataset, steps, batch=32, lr=1e-3, lr_min=1e-5, seed=0, log=None, log_every=500,
          weighted=True, group=None):
    """Adam with cosine decay on random (trajectory, macro-step) pairs, loss weighted per
    trajectory (``Dataset.w``) unless weighted=False; returns the loss history and the
    measured training throughput (samples/s, including batch assembly).  Under
    torch.distributed with several ranks every rank draws its own batches and the
    gradients are averaged each step (``dp_step``); samples/s then counts all ranks."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    g = torch.Generator(device=data.u.device).manual_seed(seed + 7919 * rank)
    hist = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(steps):
        traj = torch.randint(0, data.n, (batch,), generator=g, device=data.u.device)
        k = torch.randint(0, data.K, (batch,), generator=g, device=data.u.device)
        x, y = data.batch(traj, k)
        a = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * it / max(steps, 1)))
        w = data.w[traj].contiguous() if weighted else None
        if world > 1:
            hist.append(dp_step(net, x, y, w, float(a), group))
        else:
            hist.append(net.train_step(x, y, float(a), weights=w))
        if log and (it + 1) % log_every == 0:
            log(f"step {it + 1}/{steps} loss {np.mean(hist[-log_every:]):.4e}")
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"loss": hist, "samples_per_s": world * steps * batch / dt, "seconds": dt, "ranks": world}


def rollout(net, u0, static, n_steps):
    """Chains n_steps macro-steps from u0 [B, N, N] (metres) with per-member static
    features [B, 5, N, N]; returns u [n_steps + 1, B, N, N] (torch, metres)."""
    import torch

    us = [u0]
    u = u0
    for _ in range(n_steps):
        x = torch.cat([(u / U_SCALE).unsqueeze(1), static], dim=1).contiguous()
        u = u + DU_SCALE * net.predict(x)
        us.append(u)
    return torch.stack(us)


def _rel(a, b, dims=(-2, -1)):
    import torch

    return torch.linalg.vector_norm(a - b, dim=dims) / torch.linalg.vector_norm(b, dim=dims).clamp_min(1e-30)


def evaluate(net, data: Dataset):
    """Held-out accuracy: rel-L2 of one macro-step (of u and of the increment) from the
    solver's states, and of the full rollout from u(0) = 0, against the solver."""
    import torch

    n, K = data.n, data.K
    traj = torch.arange(n, device=data.u.device).repeat_interleave(K)
    k = torch.arange(K, device=data.u.device).repeat(n)
    x = data.inputs(traj, k)
    du_pred = DU_SCALE * net.predict(x)
    du_true = data.u[traj, k + 1] - data.u[traj, k]
    step_u = _rel(data.u[traj, k] + du_pred, data.u[traj, k + 1])
    step_du = _rel(du_pred, du_true)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    roll = rollout(net, data.u[:, 0], data.static, K)
    torch.cuda.synchronize()
    t_roll = time.perf_counter() - t0
    roll_err = _rel(roll.transpose(0, 1), data.u)                                # [n, K+1]
    return {
        "one_step_relL2_du_pooled": float(torch.linalg.vector_norm(du_pred - du_true)
                                          / torch.linalg.vector_norm(du_true)),
        "one_step_relL2_u_mean": float(step_u.mean()),
        "one_step_relL2_du_mean": float(step_du.mean()),
        "one_step_relL2_du_median": float(step_du.median()),
        "rollout_relL2_final_mean": float(roll_err[:, -1].mean()),
        "rollout_relL2_final_median": float(roll_err[:, -1].median()),
        "rollout_relL2_final_max": float(roll_err[:, -1].max()),
        "rollout_relL2_by_step": [float(v) for v in roll_err[:, 1:].mean(0).cpu()],
        "persistence_relL2_final_mean": float(_rel(data.u[:, -2], data.u[:, -1]).mean()),
        "infer_samples_per_s": n * K / t_roll,
    }


# ---------------------------------------------------------------------------
# screening
# ---------------------------------------------------------------------------

@dataclass
class ScreenReport:
    accepted: list
    solver_runs: int
    out_of_bound: int
    misfit_rejects: int
    surrogate_seconds: float
    solver_seconds: float
    checked: list = field(default_factory=list)   # (pool index, surrogate error, solver misfit, accepted)


def solve_final(specs, t_end, batch=128):
    """u(t_end) of each member from the plain solver (ensemble kernel), [n, N, N]."""
    out = np.zeros((len(specs), specs[0].N, specs[0].N), dtype=np.float32)
    for b0 in range(0, len(specs), batch):
        part = specs[b0:b0 + batch]
        sims = [simulation_for(s, t_end) for s in part]
        ens = M.Ensemble(sims)
        st = ens.step(t_end)
        if any(st):
            raise RuntimeError(f"solver failed: status {st}")
        for i, sim in enumerate(sims):
            out[b0 + i] = sim.get_field("u").T
        ens.close()
        for s in sims:
            s.close()
    return out


def _misfit(u, obs):
    return float(np.linalg.norm(u - obs) / max(np.linalg.norm(obs), 1e-30))


def screen(net, pool, obs, n_accept, tol_obs, bound, t_end, solve_batch=8, solver=None, device="cuda"):
    """Surrogate proposes, plain solver checks.  pool: MemberSpecs; obs: observed u(t_end)
    [N, N].  A proposal is accepted when the solver's u(t_end) fits obs within tol_obs
    (rel-L2) and the surrogate's prediction is within `bound` (rel-L2) of the solver's;
    otherwise it is replaced by the next proposal.  solver(specs, t_end) -> u(t_end)
    defaults to ``solve_final``."""
    import torch

    solver = solver or solve_final
    t0 = time.perf_counter()
    static = torch.from_numpy(np.stack([static_features(s) for s in pool])).to(device)
    u0 = torch.zeros((len(pool), pool[0].N, pool[0].N), device=device)
    pred = rollout(net, u0, static, int(round(t_end / MACRO_DT)))[-1].cpu().numpy()
    t_sur = time.perf_counter() - t0
    order = np.argsort([_misfit(p, obs) for p in pred])
    rep = ScreenReport([], 0, 0, 0, t_sur, 0.0)
    pos = 0
    while len(rep.accepted) < n_accept and pos < len(order):
        take = order[pos:pos + min(solve_batch, n_accept - len(rep.accepted))]
        pos += len(take)
        t1 = time.perf_counter()
        exact = solver([pool[i] for i in take], t_end)
        rep.solver_seconds += time.perf_counter() - t1
        rep.solver_runs += len(take)
        for i, u in zip(take, exact):
            e, m = _misfit(pred[i], u), _misfit(u, obs)
            ok = m <= tol_obs and e <= bound
            if e > bound:
                rep.out_of_bound += 1
            elif m > tol_obs:
                rep.misfit_rejects += 1
            if ok:
                rep.accepted.append((int(i), u))
            rep.checked.append((int(i), e, m, ok))
    return rep


def screen_without_surrogate(pool, obs, n_accept, tol_obs, t_end, seed=0, solve_batch=8, solver=None):
    """The same acceptance loop with the solver alone: candidates in random order."""
    solver = solver or solve_final
    order = np.random.default_rng(seed).permutation(len(pool))
    rep = ScreenReport([], 0, 0, 0, 0.0, 0.0)
    pos = 0
    while len(rep.accepted) < n_accept and pos < len(order):
        take = order[pos:pos + min(solve_batch, n_accept - len(rep.accepted))]
        pos += len(take)
        t1 = time.perf_counter()
        exact = solver([pool[i] for i in take], t_end)
        rep.solver_seconds += time.perf_counter() - t1
        rep.solver_runs += len(take)
        for i, u in zip(take, exact):
            m = _misfit(u, obs)
            if m <= tol_obs:
                rep.accepted.append((int(i), u))
            else:
                rep.misfit_rejects += 1
            rep.checked.append((int(i), None, m, m <= tol_obs))
    return rep


def calibration_pool(n, N, W, seed, truth_mean=21.0, truth_amp=0.5, spread=1.0):
    """A viscosity calibration problem: the truth member and n candidates that share its
    ice, lithosphere and viscosity pattern g and differ in log10 eta = m + a g, with
    m ~ U[truth_mean - spread, truth_mean + spread] and a ~ U[0.25, 0.75]; returns
    (truth, pool)."""
    truth = member_spec(seed, N, W, eta_mean=truth_mean, eta_amp=truth_amp)
    rng = np.random.default_rng(seed + 1)
    means = rng.uniform(truth_mean - spread, truth_mean + spread, n)
    amps = rng.uniform(0.25, 0.75, n)
    g = truth.meta["eta_pattern"]
    pool = [member_spec(seed + 100 + i, N, W, eta_mean=means[i], ice=truth.H, T=truth.T, eta_pattern=g,
                        eta_amp=amps[i]) for i in range(n)]
    return truth, pool


# ---------------------------------------------------------------------------
# the full-size run: 128^2 members, 10-kyr trajectories, held-out evaluation, screening
# ---------------------------------------------------------------------------

def main(argv=None):
    import argparse
    import json

    import torch

    from .fno import FNO

    ap = argparse.ArgumentParser(description="train and evaluate the macro-step surrogate")
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--W", type=float, default=1.5e6)
    ap.add_argument("--n-train", type=int, default=2000)
    ap.add_argument("--n-test", type=int, default=200)
    ap.add_argument("--t-end", type=float, default=10e3)
    ap.add_argument("--steps", type=int, default=30000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--pool", type=int, default=128)
    ap.add_argument("--accept", type=int, default=4)
    ap.add_argument("--tol", type=float, default=0.05)
    ap.add_argument("--bound", type=float, default=0.1)
    ap.add_argument("--unweighted", action="store_true")
    ap.add_argument("--out", default="surrogate_report.json")
    ap.add_argument("--save-params", default=None)
    a = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)  # noqa: E731
    rep = {"config": vars(a)}
    t0 = time.perf_counter()
    train_specs = [member_spec(s, a.N, a.W) for s in range(a.n_train)]
    test_specs = [member_spec(100000 + s, a.N, a.W) for s in range(a.n_test)]
    u_train = generate_trajectories(train_specs, a.t_end, log=log, device="cuda")
    u_test = generate_trajectories(test_specs, a.t_end, log=log, device="cuda")
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    rep["generation"] = {"seconds": t_gen,
                         "member_kyr_per_s": (a.n_train + a.n_test) * a.t_end / 1e3 / t_gen}
    data, test = Dataset(train_specs, u_train), Dataset(test_specs, u_test)
    net = FNO(S=a.N, max_batch=max(a.batch, 64), seed=0)
    hist = train(net, data, a.steps, batch=a.batch, lr=a.lr, log=log, log_every=2000, weighted=not a.unweighted)
    rep["training"] = {"samples_per_s": hist["samples_per_s"], "seconds": hist["seconds"], "steps": a.steps,
                       "loss_first_100": float(np.mean(hist["loss"][:100])),
                       "loss_last_1000": float(np.mean(hist["loss"][-1000:]))}
    log(json.dumps(rep["training"]))
    ev = evaluate(net, test)
    rep["held_out"] = ev
    log(json.dumps({k: v for k, v in ev.items() if k != "rollout_relL2_by_step"}))
    if a.save_params:
        np.save(a.save_params, net.get_params())
    truth, pool = calibration_pool(a.pool, a.N, a.W, seed=424242)
    obs = solve_final([truth], a.t_end)[0]
    t1 = time.perf_counter()
    exact = solve_final(pool, a.t_end)
    t_all = time.perf_counter() - t1
    mis = np.array([_misfit(x, obs) for x in exact])
    ws = screen(net, pool, obs, a.accept, a.tol, a.bound, a.t_end, solve_batch=a.accept)
    wo = screen_without_surrogate(pool, obs, a.accept, a.tol, a.t_end, seed=1, solve_batch=a.accept)
    rep["screening"] = {
        "pool": a.pool, "qualifying_in_pool": int((mis <= a.tol).sum()), "tol": a.tol, "bound": a.bound,
        "solver_all_pool_seconds": t_all,
        "with_surrogate": {"solver_runs": ws.solver_runs, "accepted": len(ws.accepted),
                           "out_of_bound": ws.out_of_bound, "misfit_rejects": ws.misfit_rejects,
                           "surrogate_seconds": ws.surrogate_seconds, "solver_seconds": ws.solver_seconds,
                           "accepted_solver_misfit_max": max([_misfit(u, obs) for _, u in ws.accepted], default=None),
                           "checked": [(i, e, m, ok) for i, e, m, ok in ws.checked]},
        "without_surrogate": {"solver_runs": wo.solver_runs, "accepted": len(wo.accepted),
                              "solver_seconds": wo.solver_seconds},
    }
    log(json.dumps({k: v for k, v in rep["screening"].items() if k not in ("with_surrogate",)}))
    log(json.dumps({k: v for k, v in rep["screening"]["with_surrogate"].items() if k != "checked"}))
    with open(a.out, "w") as f:
        json.dump(rep, f, indent=1)
    net.close()
    return rep


if __name__ == "__main__":
    main()
