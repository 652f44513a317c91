"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): each rank of a
multi-GPU run indexes its own shard of config-3 files (distinct seeds, rank 0
= the single-GPU workload), timings reduce to the max over ranks and bytes to
the sum, with no collective on the data path."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init()
    size_seed, base = bench.c3_shard_seeds(r)
    sizes = bench.c3_sizes(seed=size_seed, count=200, total=200 * 100_000)
    t_max = bench.allreduce_max(float(10 * (r + 1)), w)
    b_sum = bench.allreduce_sum(float(sizes.sum()), w)
    bench.barrier(w)
    seeds = [None] * w
    dist.all_gather_object(seeds, (size_seed, base))
    dist.destroy_process_group()
    Path(out_dir, f"rank{r}.json").write_text(json.dumps({
        "world": w, "t_max": t_max, "b_sum": b_sum, "mine": int(sizes.sum()), "seeds": seeds}))


def test_two_ranks_shard_files_and_reduce(tmp_path):
    if sys.platform != "linux":
        pytest.skip("gloo test runs on Linux")
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    assert all(x["world"] == world for x in res)
    assert all(x["t_max"] == 20.0 for x in res)
    total = sum(x["mine"] for x in res)
    assert all(x["b_sum"] == float(total) for x in res)
    seeds = [tuple(s) for s in res[0]["seeds"]]
    assert seeds[0] == (3, 0)  # rank 0 runs the single-GPU workload
    assert len(set(seeds)) == world  # every rank its own files
    assert res[0]["mine"] != res[1]["mine"]
