"""The surrogate's data-parallel training step (surrogate.dp_step) with two gloo ranks on
CPU: after every step the ranks hold identical parameters, equal to one process training
on the union of their batches (the all-reduced mean of equal-size per-rank mean
gradients is the gradient of the mean over the union)."""
import pathlib
import subprocess
import sys

import numpy as np

from test_shard_gloo import _free_port


def test_two_gloo_ranks_dp_step(tmp_path):
    world, port = 2, _free_port()
    script = pathlib.Path(__file__).resolve().parent / "fno_dp_rank.py"
    procs = [subprocess.Popen([sys.executable, str(script), str(r), str(world), str(port), str(tmp_path)])
             for r in range(world)]
    try:
        codes = [p.wait(timeout=240) for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert codes == [0, 0]
    views = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    assert views[0]["p"] == views[1]["p"]                   # identical on both ranks
    assert views[0]["losses"] == views[1]["losses"]
    # one process on the union of the two batches
    rng = np.random.default_rng(100)
    X = rng.standard_normal((20, 8, 5)).astype(np.float32)
    Y = rng.standard_normal((20, 8)).astype(np.float32)
    p = np.linspace(-1.0, 1.0, 5, dtype=np.float32).astype(np.float64)
    for k in range(20):
        r = X[k] @ p - Y[k]
        p = p - 0.05 * (2.0 * (X[k].T @ r) / 8)
    np.testing.assert_allclose(views[0]["p"], p, rtol=1e-5, atol=1e-6)
