"""CPU checks of the surrogate network's FP64 oracle: the FFT-based spectral convolution
against direct DFT sums, and the hand-written adjoint against central finite differences."""
import numpy as np

from oracle import fno_oracle as O


def test_spectral_conv_is_truncated_dft():
    S = 32
    rng = np.random.default_rng(0)
    v = rng.standard_normal((1, O.C, S, S))
    W = rng.standard_normal((O.KX, O.KY, O.C, O.C)) + 1j * rng.standard_normal((O.KX, O.KY, O.C, O.C))
    s, Vm = O.spectral(v, W)
    ky = O.ky_index(S)
    yy, xx = np.meshgrid(np.arange(S), np.arange(S), indexing="ij")
    sd = np.zeros_like(s)
    for a, k in enumerate(ky):
        for kx in range(O.KX):
            ph = np.exp(-2j * np.pi * (k * yy + kx * xx) / S)
            V = (v * ph).sum(axis=(-2, -1))                          # [1, C]
            assert np.abs(V - Vm[:, :, a, kx]).max() < 1e-9
            Y = V @ W[kx, a]                                          # [1, C]
            w = 1.0 if kx == 0 else 2.0
            sd += w / (S * S) * np.real(Y[:, :, None, None] * np.conj(ph))
    assert np.abs(sd - s).max() < 1e-9 * np.abs(s).max()


def test_adjoint_matches_finite_differences():
    S, B = 32, 2
    rng = np.random.default_rng(1)
    p = O.init_params(3, scale_spec=0.05)
    x = rng.standard_normal((B, 6, S, S))
    t = rng.standard_normal((B, S, S))
    q, cache = O.forward(p, x)
    _, dq = O.mse(q, t)
    g = O.backward(p, cache, dq)
    o = O.offsets()
    idx = [o["P"] + 3, o["bP"] + 5, o["layer"][0] + 7, o["layer"][1] + O.SPEC + 17,
           o["layer"][2] + O.SPEC + O.C * O.C + 3, o["layer"][3] + O.SPEC + 100, o["Q1"] + 77, o["b1"] + 9,
           o["Q2"] + 4, o["b2"], o["layer"][1] + (3 * 32 + 20) * 2048 + 1024 + 5, o["layer"][3] + 12345]
    for i in idx:
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.mse(O.forward(pp, x)[0], t)[0] - O.mse(O.forward(pm, x)[0], t)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-4 * abs(fd) + 1e-10, (i, g[i], fd)
