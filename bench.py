#!/usr/bin/env python
"""Benchmark of the LV-ELVA hot path: kyr simulated per second on the N=350 glacial
cycle (6000 km domain, seeded random viscosity / lithosphere / ice fields, elastic,
viscous and sea-surface convolutions on), fused FP32 form on one B200.

One bench step = advancing the simulation by one kyr of the glacial cycle
(consecutive segments; about 17k adaptive BS3 steps each).  `value` is kyr/s with all
inputs resident on the device (CUDA-event time on the library's stream); `e2e` is the
same metric through the public coupling API (init_integrator / step! with an
externally supplied ice field copied from host memory every step and the displacement
read back).  Also reported: the plain FP64 form (the comparison baseline), the
dominant kernel against the HBM roofline, the surrogate network's training and inference
throughput, the N=1024 high-resolution case, and the CPU oracle timed on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
import fastiso_b200 as F  # noqa: E402
import fastiso_b200.workloads as W  # noqa: E402

METRIC = "kyr simulated/s at N=350 vs plain FP64 GPU @relL2<=1e-4; ensemble member-kyr/s"
SEG_YR = 1000.0
N350 = 350
PEAKS_PATH = ROOT / "MEASURED_PEAKS.json"


def hbm_peak():
    try:
        return float(json.loads(PEAKS_PATH.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def l2_flush(dev):
    """Write 256 MiB (> 126 MB L2) between timed steps."""
    import torch

    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")
    buf.fill_(1.0)
    torch.cuda.synchronize(dev)
    del buf


def counters(sim):
    st = sim.stats()
    return {k: st[k] for k in ("nf", "naccept", "nreject", "nsparse", "segments", "gpu_ms", "executor", "grid")}


def launches_between(a, b, executor):
    """Kernels of this library launched between two counter snapshots.  Persistent
    executor: one k_persist per segment, plus 7 per host-driven right-hand side (the
    FSAL re-evaluation after an output: gate, 3 convolution, 3 RHS kernels).  Graph and
    loop executors: 3 per right-hand side, 3 per sparse update, 1 per segment start."""
    attempts = (b["naccept"] + b["nreject"]) - (a["naccept"] + a["nreject"])
    nf = b["nf"] - a["nf"]
    if executor == 0:
        return (b["segments"] - a["segments"]) + 7 * max(0, nf - 3 * attempts)
    return 3 * nf + 3 * (b["nsparse"] - a["nsparse"]) + (b["segments"] - a["segments"])


def phase_timeline(sim, integ, years=50.0):
    """Per-phase time of the persistent executor (block 0's view: the slowest block of
    the phase plus the grid barrier), from fi_trace_phases over `years` of simulation,
    outside the timed region."""
    import ctypes as C
    from fastiso_b200 import abi

    if sim.stats()["executor"] != abi.FI_EXEC_PERSIST:
        return None
    lib, h = sim.lib, sim._handle
    if lib.fi_trace_phases(h, 1):
        return None
    F.step(integ, years, True)
    ms = (C.c_double * abi.FI_NUM_PHASES)()
    cnt = (C.c_int64 * abi.FI_NUM_PHASES)()
    lib.fi_get_phase_trace(h, ms, cnt)
    lib.fi_trace_phases(h, 0)
    out = {}
    for name, t, c in zip(abi.PHASE_NAMES, ms, cnt):
        if c:
            out[name] = {"us": round(1e3 * t / c, 3), "count": int(c)}
    return out


def bytes_per_launch(nx, ny):
    """Algorithmic bytes of each fused kernel (stage-2 variants as timed): every input
    read once, every output written once, halo re-reads and twiddles not counted."""
    n = nx * ny
    NH = nx // 2 + 1
    spec = 8 * NH * ny  # complex64 half spectrum
    Mx, My = F.nextfastfft(2 * nx - 1), F.nextfastfft(2 * ny - 1)
    MH = Mx // 2 + 1
    return {
        # uprev f64, k1, D, K/(2eta), two ice snapshots, ue, dz in; S, sig_load, sig_geo out
        "k_rows_fwd": 8 * n + 4 * n * 7 + spec + 8 * n,
        "k_cols": 2 * spec + 4 * NH * ny,
        "k_rows_inv": spec + 4 * n,
        "k_conv_rows": 2 * 4 * n + 2 * 8 * MH * ny,
        "k_conv_cols": 2 * (8 * MH * ny + 8 * MH * My + 8 * MH * (ny + 2)),
        "k_conv_rows_inv": 2 * 8 * MH * (ny + 2) + 2 * 4 * n,
    }


def roofline(dev, us_per_bs3, steps_per_launch, executor, grid):
    """The persistent step kernel against the HBM roofline: algorithmic bytes of one BS3
    step (three right-hand sides, each reading its inputs once and writing its outputs
    once: rows_fwd + cols + rows_inv of bytes_per_launch) times the steps of a launch,
    over the launch's CUDA-event duration.  The per-phase kernels are timed alone with
    fi_time_kernels for reference."""
    import ctypes as C

    sim = W.config2(form="fp32", N=N350)
    sim.cfg.device = dev
    F.init_integrator(sim)
    ms = (C.c_double * 6)()
    rc = sim.lib.fi_time_kernels(sim._handle, 200, ms)
    sim.close()
    if rc:
        raise RuntimeError(f"fi_time_kernels failed ({rc})")
    names = ["k_rows_fwd", "k_cols", "k_rows_inv", "k_conv_rows", "k_conv_cols", "k_conv_rows_inv"]
    bpl = bytes_per_launch(N350, N350)
    per_step = 3 * (bpl["k_rows_fwd"] + bpl["k_cols"] + bpl["k_rows_inv"])
    peak, kind = hbm_peak()
    achieved = per_step / (us_per_bs3 * 1e-6) / 1e9
    traffic = None
    tpath = ROOT / "profiles" / "roofline_traffic.json"
    if tpath.exists():
        per = json.loads(tpath.read_text()).get("k_persist_bytes_per_bs3_step")
        if per:
            traffic = round(per * steps_per_launch)
    return {"bound": "hbm", "kernel": "k_persist" if executor == 0 else "k_rows_fwd/k_cols/k_rows_inv",
            "achieved": round(achieved, 1), "peak": peak, "peak_kind": kind, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "bytes_per_launch": round(per_step * steps_per_launch), "bytes_per_bs3_step": per_step,
            "bs3_steps_per_launch": steps_per_launch, "grid": grid,
            "note": "one member's working set is L2-resident within a launch: DRAM traffic is far below the "
                    "algorithmic bytes and the kernel is latency-bound, not HBM-bound",
            "phase_kernels_alone_ms": {k: round(v, 5) for k, v in zip(names, list(ms))}}


ENS_MEMBERS = 128
ENS_WINDOW_YR = 1000.0


def ensemble_bench(dev, rank=0, world=1):
    """Config 3: 128 members, N drawn from {64, 96, 128, 192, 256} over N x 30 km, own
    seeded viscosity fields, shared disc + random-field ice history; the persistent
    ensemble executor advances all members one window.  Under torchrun the members are
    sharded over the ranks (greedy bin-packing on N^2 log N, no communication in the time
    loop, one gather at the end) and the window's time is the slowest rank's.  Compared
    against looping the plain FP64 form member by member (sampled on 4 members, rank 0)."""
    from fastiso_b200.shard import run_shard

    members, t_ice, mod = W.config3_members(n_members=ENS_MEMBERS)
    parts = run_shard(members, t_ice, mod, ENS_WINDOW_YR, rank, world, device=dev)
    if rank != 0:
        return None
    ms = max(p["ms"] for p in parts)
    ok = all(x == 0 for p in parts for x in p["status"])
    tot_kyr, tot_ms = 0.0, 0.0
    for m in members[:4]:
        ps = W.config3_simulation(m, t_ice, mod, form="fp64")
        ps.cfg.device = dev
        ps.cfg.max_steps = 50_000_000
        pit = F.init_integrator(ps)
        F.step(pit, 50.0, True)
        F.step(pit, 200.0, True)
        tot_kyr += 0.2
        tot_ms += ps.stats()["last_gpu_ms"]
        ps.close()
    v = ENS_MEMBERS * ENS_WINDOW_YR / 1e3 / (ms / 1e3)
    plain = tot_kyr / (tot_ms / 1e3)
    # HBM roofline of k_ens: algorithmic bytes of every member's BS3 attempts in the window
    # (3 right-hand sides each: rows_fwd + cols + rows_inv of its own N) over the window's
    # device time (the slowest rank's)
    byts = 0
    for p in parts:
        for i, att in zip(p["members"], p.get("attempts", [])):
            N = members[i]["N"]
            bpl = bytes_per_launch(N, N)
            byts += 3 * att * (bpl["k_rows_fwd"] + bpl["k_cols"] + bpl["k_rows_inv"])
    peak, kind = hbm_peak()
    achieved = byts / (ms * 1e-3) / 1e9 if byts else None
    roof = {"bound": "hbm", "kernel": "k_ens", "achieved": round(achieved, 1) if achieved else None,
            "peak": peak, "peak_kind": kind, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None, "bytes_per_window": byts,
            "member_attempts": int(sum(sum(p.get("attempts", [])) for p in parts))}
    from fastiso_b200.autotune import ensemble_rule_for, tiles_for

    rule = ensemble_rule_for()
    tiles = (f"per member: h = B = clamp({rule} // N, 2, 16)" if rule is not None else
             list(tiles_for(f"ensemble:{len(parts[0]['members'])}") or F.Ensemble.DEFAULT_TILES))
    return {"value": v, "unit": "member-kyr/s", "members": ENS_MEMBERS, "ranks": world,
            "members_per_rank": [len(p["members"]) for p in parts],
            "window": f"{ENS_WINDOW_YR:g} yr after 50 yr (of config 3's 20 kyr)",
            "tiles": tiles,
            "status_ok": ok, "ms": ms,
            "plain_fp64_loop": {"value": plain, "unit": "member-kyr/s",
                                "sample": "4 members x 200 yr after 50 yr, one after another"},
            "speedup_vs_plain_loop": v / plain, "roofline": roof}


C5_WARM_YR, C5_TIMED_YR, C5_CMP_YR = 5.0, 20.0, 500.0


def config5_bench(dev):
    """Config 5: N = 1024 over 6000 km (dx ~ 5.9 km) with the config-2 generators, FP32
    form.  kyr/s over a short window after a warm-up (the full 30-kyr segment is ~50x
    longer than this run's time budget allows), the persistent kernel against the HBM
    roofline (at this size one right-hand side's algorithmic bytes, ~50 MB, no longer
    fit comfortably in L2), and rel-L2 of u against the plain FP64 form after the first
    C5_CMP_YR years."""
    sim = W.config5(form="fp32")
    sim.cfg.device = dev
    sim.cfg.max_steps = 50_000_000
    integ = F.init_integrator(sim)
    F.step(integ, C5_WARM_YR, True)
    c0 = counters(sim)
    with ClockSampler(dev) as clk:
        l2_flush(dev)
        F.step(integ, C5_TIMED_YR, True)
    c1 = counters(sim)
    ms = c1["gpu_ms"] - c0["gpu_ms"]
    attempts = (c1["naccept"] + c1["nreject"]) - (c0["naccept"] + c0["nreject"])
    n = 1024
    bpl = bytes_per_launch(n, n)
    per_step = 3 * (bpl["k_rows_fwd"] + bpl["k_cols"] + bpl["k_rows_inv"])
    peak, kind = hbm_peak()
    achieved = per_step * attempts / (ms * 1e-3) / 1e9
    u32_end = sim.get_field("u")
    sim.close()
    # accuracy: FP32 vs plain FP64 after the first C5_CMP_YR years (from t = 0)
    a = W.config5(form="fp32")
    b = W.config5(form="fp64")
    out = {}
    for name, s in (("fp32", a), ("fp64", b)):
        s.cfg.device = dev
        s.cfg.max_steps = 50_000_000
        it = F.init_integrator(s)
        F.step(it, C5_CMP_YR, True)
        out[name] = (s.get_field("u"), s.stats())
        s.close()
    ua, ub = out["fp32"][0], out["fp64"][0]
    plain_ms = out["fp64"][1]["gpu_ms"]
    return {"value": C5_TIMED_YR / 1e3 / (ms / 1e3), "unit": "kyr/s", "N": n,
            "window": f"{C5_TIMED_YR:g} yr after {C5_WARM_YR:g} yr", "bs3_steps": attempts,
            "us_per_bs3_step": 1e3 * ms / max(1, attempts),
            "rhs_evals_per_s": (c1["nf"] - c0["nf"]) / (ms / 1e3),
            "roofline": {"bound": "hbm", "kernel": "k_persist", "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "bytes_per_bs3_step": per_step},
            "plain_fp64": {"value": C5_CMP_YR / 1e3 / (plain_ms / 1e3), "unit": "kyr/s",
                           "sample": f"first {C5_CMP_YR:g} yr"},
            "relL2_u_vs_fp64": float(np.linalg.norm(ua - ub) / max(np.linalg.norm(ub), 1e-300)),
            "u_finite": bool(np.isfinite(u32_end).all()),
            "clocks": clk.summary()}


def output_bench(dev, kyr=2.0, every=100.0):
    """run! on the N = 350 workload over the first `kyr` kyr with NativeOutput every
    `every` yr (u, ue, dudt, dz_ss: 4 x 1 MB per output through the asynchronous
    staging / copy-stream pipeline) against the same run with a single output at the
    end; wall clock of the whole fi_run call, so the host side of the outputs counts."""
    res = {}
    for name, outs in (("every", list(np.arange(every, kyr * 1e3 + 1, every))), ("end_only", [kyr * 1e3])):
        sim = W.config2(form="fp32", N=N350, t_end=kyr * 1e3)
        sim.cfg.device = dev
        sim.cfg.max_steps = 20_000_000
        sim.nout.t = [float(t) for t in outs]
        sim.init_problem()
        t0 = time.perf_counter()
        F.run(sim)
        el = time.perf_counter() - t0
        assert all(np.isfinite(a).all() for a in sim.nout.out["u"])
        res[name] = {"kyr_per_s": kyr / el, "outputs": len(outs), "wall_s": el}
        sim.close()
    res["ratio"] = res["every"]["kyr_per_s"] / res["end_only"]["kyr_per_s"]
    res["note"] = (f"fi_run over 0..{kyr:g} kyr; outputs of u, ue, dudt, dz_ss every {every:g} yr vs one at the end "
                   "(each output also re-evaluates the FSAL derivative, as the reference's output callback does)")
    return res


def config2_full(dev, kyr=120.0, seg=10.0):
    """The whole N = 350 glacial cycle (120 kyr): the plain FP64 form's adaptive run
    (recorded), the FP32 form's adaptive run, and the FP32 form replaying the FP64 record;
    kyr/s of each and rel-L2 of u and dz_ss at every `seg`-kyr output (FP32 replay vs
    FP64, FP32 adaptive vs FP64)."""
    outs = [float(t) for t in np.arange(seg, kyr + 1e-9, seg) * 1e3]

    def run(form, record=False, replay=None):
        sim = W.config2(form=form, N=N350, t_end=kyr * 1e3)
        sim.cfg.device = dev
        sim.cfg.max_steps = 500_000_000
        sim.nout.t = outs
        integ = F.init_integrator(sim)
        if record:
            sim.record_steps(1 << 26)
        if replay is not None:
            sim.set_step_replay(replay)
        fields, ms = [], 0.0
        for t in outs:
            F.step(integ, t - integ.t, True)
            ms += sim.stats()["last_gpu_ms"]
            fields.append({f: sim.get_field(f) for f in ("u", "dz_ss")})
        st = sim.stats()
        rec = sim.step_record() if record else None
        sim.close()
        return fields, ms, st, rec

    f64, ms64, st64, rec = run("fp64", record=True)
    f32, ms32, st32, _ = run("fp32")
    fr, msr, _, _ = run("fp32", replay=rec)
    err = lambda a, b, f: [rel_l2(x[f], y[f]) for x, y in zip(a, b)]  # noqa: E731
    return {"kyr": kyr, "fp64": {"kyr_per_s": kyr / (ms64 / 1e3), "attempts": st64["naccept"] + st64["nreject"]},
            "fp32": {"kyr_per_s": kyr / (ms32 / 1e3), "attempts": st32["naccept"] + st32["nreject"]},
            "speedup": ms64 / ms32,
            "fp32_replay_vs_fp64": {"u": err(fr, f64, "u"), "dz_ss": err(fr, f64, "dz_ss")},
            "fp32_adaptive_vs_fp64": {"u": err(f32, f64, "u"), "dz_ss": err(f32, f64, "dz_ss")},
            "outputs_kyr": [t / 1e3 for t in outs]}


def fno_flops_per_sample(S=128, C=32, KX=16, KY=32, PW=128, nin=6, layers=4):
    """Algorithmic FLOPs of one forward pass of the surrogate per sample (the GEMMs as
    contracted, without padding): lift, per layer the DFT along x and y, the mode mixing,
    the inverse along y and x and the pointwise path, the projection."""
    S2 = S * S
    layer = (2 * C * S * 2 * KX * S + 2 * KX * C * 2 * KY * 2 * S + 2 * KX * KY * 64 * 64
             + 2 * C * KX * 2 * S * 2 * KY + 2 * S2 * C * C + 2 * C * S * S * 2 * KX)
    return 2 * S2 * C * nin + layers * layer + 2 * S2 * PW * C + 2 * S2 * PW


def fno_bench(dev, steps, warmup, S=128, B=32):
    """The surrogate's own kernels: training steps (forward, loss, backward, Adam) and
    forward passes on a synthetic batch of 32 samples of 6 x 128 x 128 (the config-4
    shape), timed with CUDA events around the synchronous calls."""
    import torch
    from fastiso_b200.fno import FNO

    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(B, 6, S, S, generator=g).cuda(dev)
    t = torch.randn(B, S, S, generator=g).cuda(dev)
    net = FNO(S=S, max_batch=B, device=dev, seed=0)
    for _ in range(warmup):
        net.train_step(x, t, 1e-4)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize(dev)
    ev[0].record()
    for _ in range(steps):
        net.train_step(x, t, 1e-4)
    ev[1].record()
    y = net.forward(x)
    for _ in range(warmup):
        net.forward(x, out=y)
    ev[2].record()
    for _ in range(steps):
        net.forward(x, out=y)
    ev[3].record()
    torch.cuda.synchronize(dev)
    net.close()
    train_ms = ev[0].elapsed_time(ev[1]) / steps
    fwd_ms = ev[2].elapsed_time(ev[3]) / steps
    f = fno_flops_per_sample(S)
    return {"train_samples_per_s": B / (train_ms / 1e3), "infer_samples_per_s": B / (fwd_ms / 1e3),
            "train_ms_per_step": train_ms, "forward_ms_per_batch": fwd_ms, "batch": B, "S": S,
            "forward_gflop_per_sample": f / 1e9,
            "forward_tflops": f * B / (fwd_ms / 1e3) / 1e12}


FP64_WINDOW_MAX_KYR = 5  # plain FP64 form and replay accuracy: the first segments of the timed window


def fp64_window(dev, warm_kyr, win_kyr):
    """The plain FP64 form on the headline workload: from t = 0, 1-kyr segments through
    the warm-up and then `win_kyr` segments of the timed window (the same segments as
    the FP32 headline).  Records every attempt (fi_record_steps) for the FP32 replay,
    times each window segment with CUDA events, keeps u, dudt and dz_ss at each window
    segment end and the state at the window start (for the CPU oracle's resume)."""
    psim = W.config2(form="fp64", N=N350)
    psim.cfg.device = dev
    psim.cfg.max_steps = 50_000_000
    integ = F.init_integrator(psim)
    psim.record_steps(1 << 23)
    seg_ms, fields, start = [], [], None
    for k in range(warm_kyr + win_kyr):
        if k == warm_kyr:
            st = psim.stats()
            start = {"t": st["t"], "nsparse": st["nsparse"],
                     "u": psim.get_field("u"), "ue": psim.get_field("ue"), "dz_ss": psim.get_field("dz_ss")}
            a0 = st["naccept"] + st["nreject"]
        F.step(integ, SEG_YR, True)
        if k >= warm_kyr:
            seg_ms.append(psim.stats()["last_gpu_ms"])
            fields.append({f: psim.get_field(f) for f in ("u", "dudt", "dz_ss")})
    st = psim.stats()
    rec = psim.step_record()
    ck = psim.checkpoint()
    psim.close()
    return {"seg_ms": seg_ms, "fields": fields, "record": rec, "start": start, "checkpoint": ck,
            "attempts": st["naccept"] + st["nreject"] - a0}


def fp32_replay_errors(dev, warm_kyr, ref):
    """The FP32 form replaying the plain FP64 form's attempt sequence from t = 0: the
    same stage times, sparse updates and accept decisions, so the difference at each
    window segment end is the FP32 arithmetic error alone."""
    sim = W.config2(form="fp32", N=N350)
    sim.cfg.device = dev
    sim.cfg.max_steps = 50_000_000
    integ = F.init_integrator(sim)
    sim.set_step_replay(ref["record"])
    errs = {f: [] for f in ("u", "dudt", "dz_ss")}
    for k in range(warm_kyr + len(ref["fields"])):
        F.step(integ, SEG_YR, True)
        if k >= warm_kyr:
            for f in errs:
                errs[f].append(rel_l2(sim.get_field(f), ref["fields"][k - warm_kyr][f]))
    # the rate at the same state: both forms evaluate dudt at the FP32 form's final u (the
    # FP64 form restored from its checkpoint at the same time, same sparse-update count)
    t_end = sim.stats()["t"] + 0.5
    p = W.config2(form="fp64", N=N350)
    p.cfg.device = dev
    p.init_problem()
    p.restore(ref["checkpoint"])
    u = sim.get_field("u")
    d32, d64 = np.zeros_like(u), np.zeros_like(u)
    F.update_diagnostics(d32, u.copy(), sim, t_end)
    F.update_diagnostics(d64, u.copy(), p, t_end)
    p.close()
    sim.close()
    return errs, rel_l2(d32, d64)


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_resumed(start, threads, seconds_target, seg=5.0, max_segs=None):
    """The FP64 oracle (the reference's CPU semantics) resumed at the window start from
    the plain FP64 form's state, stepping `seg`-yr segments until about
    `seconds_target` s of CPU work (or max_segs segments); returns (kyr/s, years)."""
    from oracle import oracle as O

    O.set_threads(threads)
    sim = W.config2(form="fp64", N=N350)
    ref = O.oracle_for(sim)
    ref.init()
    F_ = lambda a: np.asarray(a, dtype=np.float64).ravel(order="F")  # noqa: E731
    ref.resume(start["t"], start["nsparse"], F_(start["u"]), F_(start["ue"]), F_(start["dz_ss"]))
    yrs, used, n = 0.0, 0.0, 0
    while used < seconds_target and (max_segs is None or n < max_segs):
        t0 = time.perf_counter()
        ref.step(seg)
        used += time.perf_counter() - t0
        yrs += seg
        n += 1
    ref.close()
    return yrs / 1e3 / used, yrs


def config_block(warm_kyr, world):
    """The workload description shared by both arms (the reference arm times the same
    window of the same run)."""
    return {"workload": "config2 glacial cycle N=350 over 6000 km, 121 ice snapshots, "
                        "elastic+viscous+sea-surface, BS3 reltol=Float64(1f-5)",
            "window_start_kyr": warm_kyr,
            "parallelism": "replicas" if world > 1 else "single"}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU semantics (the FP64 oracle port, OpenMP over
    all host cores) on the same window of the same run as the GPU arm: the run is
    brought to the window start (t = warmup kyr) by the plain FP64 GPU form (outside
    the timed region), the oracle resumes from that state, and each step is a bounded
    5-yr sample of the window; rank 0 only."""
    if rank != 0:
        return
    from oracle import oracle as O

    warm = args.warmup
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    seg = 5.0
    sim = W.config2(form="fp64", N=N350)
    ref = O.oracle_for(sim)
    ref.init()
    if warm > 0:
        import torch

        dev = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(dev)
        p = W.config2(form="fp64", N=N350)
        p.cfg.device = dev
        p.cfg.max_steps = 50_000_000
        integ = F.init_integrator(p)
        for _ in range(warm):
            F.step(integ, SEG_YR, True)
        st = p.stats()
        F_ = lambda a: np.asarray(a, dtype=np.float64).ravel(order="F")  # noqa: E731
        ref.resume(st["t"], st["nsparse"], F_(p.get_field("u")), F_(p.get_field("ue")), F_(p.get_field("dz_ss")))
        p.close()
    else:
        ref.init_integrator([])
    t_start = ref.stats()["t"]
    for _ in range(args.warmup):
        ref.step(seg)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.step(seg)
    el = time.perf_counter() - t0
    ref.close()
    v = args.steps * seg / 1e3 / el
    sample = (f"{args.steps} x {seg:g} yr of config2 N=350 from t = {t_start / 1e3:g} kyr + {args.warmup} x "
              f"{seg:g} yr (the oracle resumed from the plain FP64 GPU form's state at the window start)")
    line = {"metric": METRIC, "value": v, "unit": "kyr/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded fields)",
            "impl": "reference",
            "config": config_block(warm, world),
            "cpu_baseline": {"value": v, "unit": "kyr/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "kyr/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_gpu(args, rank, world, dev):
    import torch

    warm = args.warmup
    # ---- headline: fused FP32 form, inputs resident ------------------------------
    sim = W.config2(form="fp32", N=N350)
    sim.cfg.device = dev
    sim.cfg.max_steps = 20_000_000
    integ = F.init_integrator(sim)
    for _ in range(warm):
        F.step(integ, SEG_YR, True)
    c0 = counters(sim)
    step_ms = []
    with ClockSampler(dev) as clk:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        for _ in range(args.steps):
            l2_flush(dev)
            F.step(integ, SEG_YR, True)
            step_ms.append(sim.stats()["last_gpu_ms"])
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()
    c1 = counters(sim)
    u_end = sim.get_field("u")
    phases = phase_timeline(sim, integ) if rank == 0 else None
    sim.close()
    ens = ensemble_bench(dev, rank, world)
    t_total = float(sum(step_ms))
    if world > 1:
        tt = torch.tensor([t_total], dtype=torch.float64, device=f"cuda:{dev}")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_total = float(tt.item())
    kyr = args.steps * SEG_YR / 1e3
    value = world * kyr / (t_total / 1e3)
    attempts = (c1["naccept"] + c1["nreject"]) - (c0["naccept"] + c0["nreject"])
    launches = launches_between(c0, c1, c1["executor"])
    if rank != 0:
        return
    assert np.isfinite(u_end).all()
    # ---- e2e: the public API with host buffers, the same time-interpolated forcing ----
    # per step: the state u uploaded from pinned host memory (integrator.u .= u, which
    # makes the next step re-evaluate its FSAL derivative), step!(1 kyr), u read back
    # into pinned host memory
    esim = W.config2(form="fp32", N=N350)
    esim.cfg.device = dev
    esim.cfg.max_steps = 20_000_000
    einteg = F.init_integrator(esim)
    n = N350 * N350
    u_pin = torch.empty(n, dtype=torch.float64, pin_memory=True)
    u_np = u_pin.numpy()
    lib, hnd = esim.lib, esim._handle
    from fastiso_b200 import abi

    def e2e_step():
        esim._check(lib.fi_set_field(hnd, abi.FIELDS["u"], abi.dptr(u_np), n), "set u")
        esim._check(lib.fi_step(hnd, SEG_YR), "fi_step")
        esim._check(lib.fi_get_field(hnd, abi.FIELDS["u"], abi.dptr(u_np), n), "get u")

    esim._check(lib.fi_get_field(hnd, abi.FIELDS["u"], abi.dptr(u_np), n), "get u")
    for _ in range(warm):
        e2e_step()
    e2e_el = 0.0
    for _ in range(args.steps):
        l2_flush(dev)
        t0 = time.perf_counter()
        e2e_step()
        e2e_el += time.perf_counter() - t0
    e2e_val = kyr / e2e_el
    assert np.isfinite(u_np).all()
    esim.close()
    # ---- plain FP64 form on the same window; FP32 replay of its attempt sequence ----
    nwin = min(args.steps, FP64_WINDOW_MAX_KYR)
    p64 = fp64_window(dev, warm, nwin)
    plain_kyr_s = nwin / (sum(p64["seg_ms"]) / 1e3)
    fp32_same = nwin / (sum(step_ms[:nwin]) / 1e3)
    replay, rate_err = fp32_replay_errors(dev, warm, p64)
    acc = {"relL2_u_vs_fp64": max(replay["u"]), "relL2_dz_ss_vs_fp64": max(replay["dz_ss"]),
           "relL2_dudt_vs_fp64": rate_err, "relL2_dudt_trajectory_vs_fp64": max(replay["dudt"])}
    # ---- roofline of the dominant kernel ----------------------------------------
    seg = max(1, c1["segments"] - c0["segments"])
    roof = roofline(dev, 1e3 * t_total / max(1, attempts), attempts / seg, c1["executor"], c1["grid"])
    # ---- the surrogate network and the N = 1024 case (outside the timed region) ----
    surrogate = fno_bench(dev, 20, max(3, args.warmup))
    config5 = config5_bench(dev)
    outputs = output_bench(dev)
    # ---- CPU baseline: the oracle resumed at the window start --------------------
    cores = os.cpu_count() or 1
    cpu_all, yrs_all = oracle_resumed(p64["start"], cores, 12.0)
    cpu_one, yrs_one = oracle_resumed(p64["start"], 1, 8.0, seg=1.0)
    win = f"t = {warm}..{warm + nwin} kyr"
    line = {
        "metric": METRIC, "value": value, "unit": "kyr/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 state)",
        "data": "synthetic (seeded Gaussian random fields)",
        "config": config_block(warm, world),
        "step": f"{SEG_YR:g} yr of simulated time (consecutive segments from t = {warm} kyr)",
        "l2": "256 MiB written between timed steps; one member's working set (~15 MB) is L2-resident within a step",
        "bs3_steps_per_bench_step": attempts / args.steps,
        "us_per_bs3_step": 1e3 * t_total / max(1, attempts),
        "rhs_evals_per_s": (c1["nf"] - c0["nf"]) / (t_total / 1e3),
        "accuracy": dict(acc, window=win, method="FP32 form replaying the plain FP64 form's recorded attempt "
                                               "sequence (dt and accept decision of every attempt) from t = 0; "
                                               "u, dz_ss: rel-L2 at every 1-kyr segment end, max over the window; "
                                               "dudt: both forms' rate at the same state (the FP32 final u); "
                                               "dudt_trajectory: the rate along each form's own trajectory, "
                                               "which the stiffest modes (~140/yr near the viscosity minimum) "
                                               "amplify from the u difference",
                         per_segment={f: [float(x) for x in e] for f, e in replay.items()}),
        **acc,
        "plain_fp64": {"value": plain_kyr_s, "unit": "kyr/s", "window": win,
                       "ms_per_bs3_step": sum(p64["seg_ms"]) / max(1, p64["attempts"]),
                       "fp32_same_window": fp32_same},
        "speedup_vs_plain_fp64": fp32_same / plain_kyr_s,
        "ensemble": ens,
        "surrogate": surrogate,
        "config5": config5,
        "output_pipeline": outputs,
        "e2e": {"value": e2e_val, "unit": "kyr/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "path": "per step: fi_set_field(u) from pinned host memory -> fi_step(1 kyr, the resident "
                        "time-interpolated ice history) -> fi_get_field(u) into pinned host memory; wall clock"},
        "gpu_launches": int(launches),
        "phases": phases,
        "roofline": roof,
        "cpu_baseline": {"value": cpu_all, "unit": "kyr/s", "cores": cores, "kind": "port",
                         "sample": f"FP64 oracle (C, OpenMP) resumed at t = {warm} kyr from the plain FP64 form's "
                                   f"state, {yrs_all:g} yr",
                         "single_thread": {"value": cpu_one, "unit": "kyr/s", "cores": 1,
                                           "sample": f"the same, 1 thread, {yrs_one:g} yr"}},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fused", choices=["fused", "reference"])
    ap.add_argument("--profile-ensemble", action="store_true",
                    help="config-3 ensemble (--members, default 16; --years, default 20) for an ncu capture of k_ens")
    ap.add_argument("--members", type=int, default=16)
    ap.add_argument("--years", type=float, default=20.0)
    ap.add_argument("--profile", action="store_true",
                    help="only a short fused N=350 segment (10 yr warm-up + 5 yr) for ncu captures")
    ap.add_argument("--fno", action="store_true",
                    help="only the surrogate network's training and inference throughput (128^2, batch 32)")
    ap.add_argument("--profile-config5", action="store_true",
                    help="N=1024: 5 yr warm-up launch, then one 0.2-yr launch of k_persist (ncu capture target)")
    ap.add_argument("--config5", action="store_true",
                    help="only the N=1024 high-resolution case (short window, roofline, rel-L2 vs FP64)")
    ap.add_argument("--config2-full", action="store_true",
                    help="the whole 120-kyr N=350 cycle: plain FP64 (recorded), FP32 adaptive, FP32 replay")
    ap.add_argument("--outputs", action="store_true",
                    help="only the output-pipeline leg (run! with outputs every 100 yr vs one output)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.profile_ensemble:
        members, t_ice, mod = W.config3_members(n_members=ENS_MEMBERS)
        members = members[:args.members]
        sims = [W.config3_simulation(m, t_ice, mod, form="fp32") for m in members]
        for sm in sims:
            sm.cfg.device = local
        ens = F.Ensemble(sims)
        ens.step(args.years)
        print(json.dumps({"profile_case": f"config3 {len(sims)} members, {args.years:g} yr", "ms": ens.last_gpu_ms,
                          "steps": [sm.stats()["naccept"] + sm.stats()["nreject"] for sm in sims]}))
        ens.close()
        return
    if args.fno:
        print(json.dumps({"fno": fno_bench(local, args.steps, args.warmup)}), flush=True)
        return
    if args.config5:
        print(json.dumps({"config5": config5_bench(local)}), flush=True)
        return
    if args.config2_full:
        print(json.dumps({"config2_full": config2_full(local)}), flush=True)
        return
    if args.outputs:
        print(json.dumps({"output_pipeline": output_bench(local)}), flush=True)
        return
    if args.profile_config5:
        sim = W.config5(form="fp32")
        sim.cfg.device = local
        integ = F.init_integrator(sim)
        F.step(integ, 5.0, True)
        F.step(integ, 0.2, True)
        print(json.dumps({"profile_case": "config5 N=1024 fp32, 5 yr + 0.2 yr", "stats": sim.stats()}))
        return
    if args.profile:
        sim = W.config2(form="fp32", N=N350)
        sim.cfg.device = local
        integ = F.init_integrator(sim)
        F.step(integ, 10.0, True)
        F.step(integ, 5.0, True)
        print(json.dumps({"profile_case": "config2 N=350 fp32, 15 yr", "stats": sim.stats()}))
        return
    try:
        run_gpu(args, rank, world, local)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
