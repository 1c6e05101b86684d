"""One rank of the two-process gloo test of the surrogate's data-parallel step
(tests/test_fno_dp_gloo.py).  A linear least-squares model on the CPU stands in for the
network: it has the FNO handle's training interface (loss_backward, grads_tensor, adam),
so the gradient averaging and the parameter agreement across ranks are what is tested.
argv: rank world port out_dir."""
import os
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from fastiso_b200.surrogate import dp_step  # noqa: E402


class LinearNet:
    """y = x . p (per sample, x [B, n]); mean-squared loss; plain gradient descent."""

    def __init__(self, n):
        self.p = torch.linspace(-1.0, 1.0, n, dtype=torch.float32)
        self.g = torch.zeros(n, dtype=torch.float32)

    def loss_backward(self, x, y, w=None):
        r = x @ self.p - y
        self.g.copy_(2.0 * (x.T @ r) / x.shape[0])
        return float((r * r).mean())

    def grads_tensor(self):
        return self.g

    def adam(self, lr):
        self.p -= lr * self.g


rank, world, port, out_dir = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
os.environ["MASTER_ADDR"] = "127.0.0.1"
os.environ["MASTER_PORT"] = str(port)
dist.init_process_group("gloo", rank=rank, world_size=world)
rng = np.random.default_rng(100)                       # same data on every rank, sliced per rank
X = torch.from_numpy(rng.standard_normal((20, 8, 5)).astype(np.float32))
Y = torch.from_numpy(rng.standard_normal((20, 8)).astype(np.float32))
net = LinearNet(5)
losses = []
for k in range(20):
    xb, yb = X[k, rank * 4:(rank + 1) * 4], Y[k, rank * 4:(rank + 1) * 4]
    losses.append(dp_step(net, xb, yb, None, 0.05))
dist.barrier()
dist.destroy_process_group()
(pathlib.Path(out_dir) / f"rank{rank}.txt").write_text(repr({"p": net.p.tolist(), "losses": losses}))
