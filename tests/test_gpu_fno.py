"""The surrogate network's CUDA forward and backward passes (fi_fno_*) against the FP64
oracle (oracle/fno_oracle.py, whose adjoint the CPU tests check by finite differences).

Tolerances: every operand of the tensor-core GEMMs is BF16 (8-bit mantissa, relative
rounding 2^-9) with FP32 accumulation, over a lift, four Fourier layers and a two-layer
projection; the outputs agree with FP64 to about 1 % and the gradients to a few %.
"""
import numpy as np
import pytest

from oracle import fno_oracle as O

pytestmark = pytest.mark.gpu

FWD_TOL = 3e-2   # rel-L2 of the network output
GRAD_TOL = 6e-2  # rel-L2 of each parameter group's gradient


def _groups():
    o = O.offsets()
    g = {"P": (o["P"], o["bP"]), "bP": (o["bP"], o["bP"] + O.C)}
    for l in range(O.NLAYER):
        b = o["layer"][l]
        g[f"W{l}"] = (b, b + O.SPEC)
        g[f"Wloc{l}"] = (b + O.SPEC, b + O.SPEC + O.C * O.C)
        g[f"bloc{l}"] = (b + O.SPEC + O.C * O.C, b + O.LAYER)
    g.update({"Q1": (o["Q1"], o["b1"]), "b1": (o["b1"], o["Q2"]), "Q2": (o["Q2"], o["b2"]),
              "b2": (o["b2"], o["total"])})
    return g


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


def _net(S, B, seed, scale_spec=0.05):
    from fastiso_b200.fno import FNO

    net = FNO(S=S, max_batch=B, seed=seed)
    p = O.init_params(seed, scale_spec=scale_spec).astype(np.float32)
    net.set_params(p)
    return net, p.astype(np.float64)


@pytest.mark.parametrize("S,B", [(32, 4), (64, 3), (128, 2)])
def test_forward_matches_oracle(torch, S, B):
    net, p = _net(S, B, seed=S + B)
    rng = np.random.default_rng(S)
    x = rng.standard_normal((B, 6, S, S)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    q, _ = O.forward(p, x)
    assert np.isfinite(y).all()
    assert _rel(y, q) < FWD_TOL, _rel(y, q)
    net.close()


def test_default_init_round_trip(torch):
    from fastiso_b200.fno import FNO

    net = FNO(S=32, max_batch=2, seed=7)
    p = net.get_params()
    assert p.size == O.num_params()
    o = O.offsets()
    spec = p[o["layer"][0]:o["layer"][0] + O.SPEC]
    assert 0 <= spec.min() and spec.max() <= 1.0 / (O.C * O.C)
    net.set_params(p * 2)
    assert np.array_equal(net.get_params(), p * 2)
    net.close()


@pytest.mark.parametrize("S,B", [(32, 4), (128, 2)])
def test_gradients_match_oracle(torch, S, B):
    net, p = _net(S, B, seed=11 + S)
    rng = np.random.default_rng(100 + S)
    x = rng.standard_normal((B, 6, S, S)).astype(np.float32)
    dy = rng.standard_normal((B, S, S)).astype(np.float32)
    net.forward(torch.from_numpy(x).cuda())
    net.backward(torch.from_numpy(dy).cuda())
    g = net.get_grads()
    _, cache = O.forward(p, x)
    gref = O.backward(p, cache, dy)
    bad = {}
    for name, (a, b) in _groups().items():
        r = _rel(g[a:b], gref[a:b])
        if not r < GRAD_TOL:
            bad[name] = r
    assert not bad, bad
    net.close()


def test_train_step_loss_and_descent(torch):
    S, B = 32, 8
    net, p = _net(S, B, seed=5)
    rng = np.random.default_rng(9)
    x = torch.from_numpy(rng.standard_normal((B, 6, S, S)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((B, S, S)).astype(np.float32)).cuda()
    q, _ = O.forward(p, x.cpu().numpy())
    want, _ = O.mse(q, t.cpu().numpy())
    losses = [net.train_step(x, t, 1e-3) for _ in range(30)]
    assert abs(losses[0] - want) / want < 2 * FWD_TOL
    assert losses[-1] < 0.9 * losses[0], losses
    net.close()


def test_weighted_loss_matches_oracle(torch):
    S, B = 32, 4
    net, p = _net(S, B, seed=21)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((B, 6, S, S)).astype(np.float32)
    t = rng.standard_normal((B, S, S)).astype(np.float32)
    w = np.array([0.5, 2.0, 1.0, 0.1], dtype=np.float32)
    loss = net.train_step(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), 0.0,
                          weights=torch.from_numpy(w).cuda())
    q, cache = O.forward(p, x)
    want, dq = O.mse(q, t, w)
    assert abs(loss - want) / want < 2 * FWD_TOL
    g = net.get_grads()   # gradients of this step (lr 0 leaves the parameters)
    gref = O.backward(p, cache, dq)
    for name in ("W0", "Wloc2", "Q1", "b2"):
        a, b = _groups()[name]
        assert _rel(g[a:b], gref[a:b]) < GRAD_TOL, name
    net.close()


def test_batch_limits(torch):
    from fastiso_b200 import abi
    from fastiso_b200.fno import FNO

    net = FNO(S=32, max_batch=2)
    x = torch.zeros((3, 6, 32, 32), device="cuda")
    with pytest.raises(abi.FiError):
        net.forward(x)
    y = net.predict(x)
    assert y.shape == (3, 32, 32)
    with pytest.raises(abi.FiError):
        net.backward(torch.zeros((2, 32, 32), device="cuda"))  # the last chunk had B = 1
    net.backward(torch.zeros((1, 32, 32), device="cuda"))
    net.close()


def test_split_step_matches_train_step(torch):
    """loss_backward + adam (the data-parallel split) is train_step, and grads_tensor is a
    zero-copy view of the gradient vector."""
    S, B = 32, 4
    a, p = _net(S, B, seed=31)
    b, _ = _net(S, B, seed=31)
    rng = np.random.default_rng(12)
    x = torch.from_numpy(rng.standard_normal((B, 6, S, S)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((B, S, S)).astype(np.float32)).cuda()
    w = torch.tensor([1.0, 0.5, 2.0, 1.5], device="cuda")
    la = a.train_step(x, t, 1e-3, weights=w)
    lb = b.loss_backward(x, t, weights=w)
    g = b.grads_tensor()
    assert g.shape == (b.n_params,) and g.is_cuda
    np.testing.assert_array_equal(g.cpu().numpy(), b.get_grads())
    b.adam(1e-3)
    assert abs(la - lb) <= 1e-6 * abs(la)
    pa, pb = a.get_params(), b.get_params()
    assert _rel(pb, pa.astype(np.float64)) < 1e-6
    from fastiso_b200.surrogate import dp_step

    dp_step(b, x, t, w, 1e-3)          # one rank: no collective, the same update
    a.train_step(x, t, 1e-3, weights=w)
    assert _rel(b.get_params(), a.get_params().astype(np.float64)) < 1e-6
    a.close()
    b.close()
