"""The benchmark's multi-GPU path on the CPU: replicas (one job per rank, no collective on the data
path) whose timing is the slowest rank's, taken with a max-reduction over gloo, world size 2."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_s = 0.1 * (rank + 1)  # rank 1 is the slower replica
    slowest = bench.rank_max(dist, local_s)
    value = bench.replica_throughput(world, 1000, 4, slowest)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{slowest!r} {value!r}\n")


def test_replicas_take_the_slowest_rank_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    for slowest, value in got:
        assert float(slowest) == 0.2
        assert abs(float(value) - world * 1000 * 4 / 0.2) < 1e-6


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(None, 0.25) == 0.25
    assert bench.replica_throughput(1, 1000, 4, 0.5) == 8000.0
