"""Ensemble sharding: the partition is complete, disjoint, balanced and the same on
every rank; two gloo ranks on CPU gather their results (the multi-GPU path without
GPUs: no collective runs inside the time loop, one gather at the end)."""
import pathlib
import socket
import sys

import subprocess

from fastiso_b200.shard import member_cost, shard_members


def test_partition_complete_and_balanced():
    import numpy as np

    rng = np.random.default_rng(2024)
    sizes = list(rng.choice([64, 96, 128, 192, 256], size=128))
    for world in (1, 2, 3, 4, 8):
        parts = shard_members(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(member_cost(sizes[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= member_cost(max(sizes)) + 1e-6
        assert parts == shard_members(sizes, world)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_gather(tmp_path):
    sizes = [64, 256, 96, 128, 192, 64, 256, 128, 96]
    world, port = 2, _free_port()
    script = pathlib.Path(__file__).resolve().parent / "gloo_rank.py"
    procs = [subprocess.Popen([sys.executable, str(script), str(r), str(world), str(port), str(tmp_path),
                               ",".join(map(str, sizes))]) for r in range(world)]
    try:
        codes = [p.wait(timeout=240) for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert codes == [0, 0]
    views = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    assert views[0] == views[1]
    got = sorted(i for part in views[0] for i in part["members"])
    assert got == list(range(len(sizes)))
    assert [p["rank"] for p in views[0]] == [0, 1]


def test_stiffness_weighted_partition():
    import numpy as np

    """Stiffer members (lower minimum viscosity) cost more; the partition balances the
    weighted cost and the weighted greedy bound holds."""
    from fastiso_b200.shard import stiffness_rate

    D = 6.6e10 * 100e3**3 / (12 * (1 - 0.28**2))
    assert stiffness_rate(1e19, D, 30e3) > 100 * stiffness_rate(1e21, D, 30e3) * 0.99
    rng = np.random.default_rng(3)
    sizes = list(rng.choice([64, 96, 128, 192, 256], size=40))
    rates = list(10.0 ** rng.uniform(-1.0, 1.0, size=40))
    for world in (1, 2, 3, 8):
        parts = shard_members(sizes, world, rates)
        assert sorted(i for p in parts for i in p) == list(range(40))
        loads = [sum(member_cost(sizes[i], rates[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(member_cost(n, r) for n, r in zip(sizes, rates)) + 1e-6
