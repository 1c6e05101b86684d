"""One rank of the two-process gloo sharding test (tests/test_shard_gloo.py).
argv: rank world port out_dir sizes(comma-separated)."""
import os
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import __graft_entry__  # noqa: E402

__graft_entry__.load_package()
import torch.distributed as dist  # noqa: E402

from fastiso_b200.shard import gather_results, shard_members  # noqa: E402

rank, world, port, out_dir = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
sizes = [int(v) for v in sys.argv[5].split(",")]
os.environ["MASTER_ADDR"] = "127.0.0.1"
os.environ["MASTER_PORT"] = str(port)
dist.init_process_group("gloo", rank=rank, world_size=world)
mine = shard_members(sizes, world)[rank]
res = gather_results({"rank": rank, "members": mine, "status": [0] * len(mine)}, world)
dist.barrier()
dist.destroy_process_group()
(pathlib.Path(out_dir) / f"rank{rank}.txt").write_text(repr(res))
