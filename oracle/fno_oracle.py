"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the surrogate network.

The checker of the ``fi_fno_*`` CUDA kernels (fastisostasy.jl_b200/csrc/fno.cu).  Only
tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import it; the product path
never does.

The network has no counterpart in FastIsostasy.jl; this module defines it.  It is the
Fourier neural operator of Li et al. (2021, "Fourier Neural Operator for Parametric Partial
Differential Equations"): lift, four Fourier layers, projection.  The spectral convolution is
written here with numpy's FFT (``rfft2`` over (y, x), x the half axis; ``irfft2`` back),
independently of the CUDA code's truncated-DFT GEMMs, and its adjoint by hand:

* forward   s = irfft2(P(W . R(v))),  R = rfft2 restricted to kx < 16, ky in {0..15, S-16..S-1},
  P = zero padding back to the half spectrum;
* adjoint   dY = (w_kx / S^2) rfft2(ds)[modes] (w = 1 at kx = 0, else 2),
            dV = sum_co dY conj(W),  dW = sum_b dY conj(V),
            dv = S^2 Re(ifft2(pad(dV))).

Parameter vector layout (``offsets``) is the one include/fastiso_b200.h documents.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

C, KX, KY, NIN, PW, NLAYER = 32, 16, 32, 6, 128, 4
NM = KX * KY
SPEC = NM * 2 * C * C
LAYER = SPEC + C * C + C


def offsets():
    o = {"P": 0, "bP": C * NIN}
    p = o["bP"] + C
    o["layer"] = []
    for _ in range(NLAYER):
        o["layer"].append(p)
        p += LAYER
    o["Q1"] = p
    o["b1"] = p + PW * C
    o["Q2"] = o["b1"] + PW
    o["b2"] = o["Q2"] + PW
    o["total"] = o["b2"] + 1
    return o


def num_params():
    return offsets()["total"]


def ky_index(S):
    return np.array([k if k < 16 else S - KY + k for k in range(KY)])


def unpack(p):
    """Flat parameter vector -> dict of arrays (views into a float64 copy)."""
    p = np.asarray(p, dtype=np.float64)
    o = offsets()
    d = {"P": p[o["P"]:o["P"] + C * NIN].reshape(C, NIN), "bP": p[o["bP"]:o["bP"] + C]}
    d["W"], d["Wloc"], d["bloc"] = [], [], []
    for l in range(NLAYER):
        b = o["layer"][l]
        w = p[b:b + SPEC].reshape(KX, KY, 2, C, C)       # [kx][kyi][re/im][ci][co]
        d["W"].append(w[:, :, 0] + 1j * w[:, :, 1])      # complex [kx][kyi][ci][co]
        d["Wloc"].append(p[b + SPEC:b + SPEC + C * C].reshape(C, C))   # [co][ci]
        d["bloc"].append(p[b + SPEC + C * C:b + LAYER])
    d["Q1"] = p[o["Q1"]:o["Q1"] + PW * C].reshape(PW, C)
    d["b1"] = p[o["b1"]:o["b1"] + PW]
    d["Q2"] = p[o["Q2"]:o["Q2"] + PW]
    d["b2"] = p[o["b2"]]
    return d


def gelu(a):
    return 0.5 * a * (1.0 + erf(a / np.sqrt(2.0)))


def gelu_grad(a):
    return 0.5 * (1.0 + erf(a / np.sqrt(2.0))) + a * np.exp(-0.5 * a * a) / np.sqrt(2.0 * np.pi)


def spectral(v, W):
    """v [B, C, S, S] (y, x) real; W complex [KX, KY, C, C] -> (s, modes of v)."""
    S = v.shape[-1]
    ky = ky_index(S)
    Vm = np.fft.rfft2(v)[:, :, ky, :KX]                          # [B, C, KY, KX]
    Y = np.einsum("bcyx,xyco->boyx", Vm, W)
    full = np.zeros(v.shape[:2] + (S, S // 2 + 1), dtype=np.complex128)
    full[:, :, ky, :KX] = Y
    return np.fft.irfft2(full, s=(S, S)), Vm


def spectral_adjoint(ds, Vm, W):
    """ds [B, C, S, S] -> (dv, dW complex [KX, KY, C, C])."""
    S = ds.shape[-1]
    ky = ky_index(S)
    w = np.where(np.arange(KX) == 0, 1.0, 2.0) / (S * S)
    dY = np.fft.rfft2(ds)[:, :, ky, :KX] * w                    # [B, C, KY, KX]
    dW = np.einsum("boyx,bcyx->xyco", dY, np.conj(Vm))
    dV = np.einsum("boyx,xyco->bcyx", dY, np.conj(W))
    full = np.zeros(ds.shape, dtype=np.complex128)
    full[:, :, ky, :KX] = dV
    dv = S * S * np.real(np.fft.ifft2(full))
    return dv, dW


def forward(params, x):
    """params: flat vector; x [B, 6, S, S] -> (q [B, S, S], cache)."""
    d = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    v = np.einsum("ci,biyx->bcyx", d["P"], x) + d["bP"][None, :, None, None]
    cache = {"x": x, "v": [v], "z": [], "Vm": []}
    for l in range(NLAYER):
        s, Vm = spectral(v, d["W"][l])
        z = s + np.einsum("oc,bcyx->boyx", d["Wloc"][l], v) + d["bloc"][l][None, :, None, None]
        v = gelu(z) if l < NLAYER - 1 else z
        cache["z"].append(z)
        cache["Vm"].append(Vm)
        cache["v"].append(v)
    a = np.einsum("jc,bcyx->bjyx", d["Q1"], v) + d["b1"][None, :, None, None]
    q = np.einsum("j,bjyx->byx", d["Q2"], gelu(a)) + d["b2"]
    cache["a"] = a
    return q, cache


def backward(params, cache, dq):
    """Gradient of sum(dq * q) with respect to the flat parameter vector."""
    d = unpack(params)
    o = offsets()
    g = np.zeros(o["total"])
    dq = np.asarray(dq, dtype=np.float64)
    a, x = cache["a"], cache["x"]
    h = gelu(a)
    v4 = cache["v"][NLAYER]
    g[o["b2"]] = dq.sum()
    g[o["Q2"]:o["Q2"] + PW] = np.einsum("byx,bjyx->j", dq, h)
    da = dq[:, None] * d["Q2"][None, :, None, None] * gelu_grad(a)
    g[o["b1"]:o["b1"] + PW] = da.sum(axis=(0, 2, 3))
    g[o["Q1"]:o["Q1"] + PW * C] = np.einsum("bjyx,bcyx->jc", da, v4).ravel()
    dv = np.einsum("bjyx,jc->bcyx", da, d["Q1"])
    for l in reversed(range(NLAYER)):
        z, v = cache["z"][l], cache["v"][l]
        dz = dv * gelu_grad(z) if l < NLAYER - 1 else dv
        b = o["layer"][l]
        g[b + SPEC + C * C:b + LAYER] = dz.sum(axis=(0, 2, 3))
        g[b + SPEC:b + SPEC + C * C] = np.einsum("boyx,bcyx->oc", dz, v).ravel()
        dvs, dW = spectral_adjoint(dz, cache["Vm"][l], d["W"][l])
        w = np.stack([dW.real, dW.imag], axis=2)           # [kx][kyi][2][ci][co]
        g[b:b + SPEC] = w.ravel()
        dv = dvs + np.einsum("oc,boyx->bcyx", d["Wloc"][l], dz)
    g[o["bP"]:o["bP"] + C] = dv.sum(axis=(0, 2, 3))
    g[o["P"]:o["P"] + C * NIN] = np.einsum("bcyx,biyx->ci", dv, x).ravel()
    return g


def mse(q, target, w=None):
    """Mean-squared error (per-sample weights w [B] if given) and its gradient w.r.t. q."""
    e = np.asarray(q, dtype=np.float64) - target
    wb = np.ones(e.shape[0]) if w is None else np.asarray(w, dtype=np.float64)
    we = wb[:, None, None] * e
    return float(np.mean(we * e)), 2.0 * we / e.size


def init_params(seed=0, scale_spec=None):
    """An initialisation for CPU-only tests (the CUDA library draws its own)."""
    rng = np.random.default_rng(seed)
    o = offsets()
    p = np.zeros(o["total"])
    u = lambda n, a: rng.uniform(-a, a, n)  # noqa: E731
    p[o["P"]:o["P"] + C * NIN] = u(C * NIN, 1 / np.sqrt(NIN))
    p[o["bP"]:o["bP"] + C] = u(C, 1 / np.sqrt(NIN))
    for l in range(NLAYER):
        b = o["layer"][l]
        p[b:b + SPEC] = rng.uniform(0, scale_spec or 1.0 / (C * C), SPEC)
        p[b + SPEC:b + SPEC + C * C] = u(C * C, 1 / np.sqrt(C))
        p[b + SPEC + C * C:b + LAYER] = u(C, 1 / np.sqrt(C))
    p[o["Q1"]:o["Q1"] + PW * C] = u(PW * C, 1 / np.sqrt(C))
    p[o["b1"]:o["b1"] + PW] = u(PW, 1 / np.sqrt(C))
    p[o["Q2"]:o["Q2"] + PW] = u(PW, 1 / np.sqrt(PW))
    p[o["b2"]] = u(1, 1 / np.sqrt(PW))[0]
    return p
