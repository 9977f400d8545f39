"""bench.py's multi-process plumbing on CPU: two gloo ranks take the same collectives in the same order,
the timing is the max over ranks and the whole-job value counts every rank's replica."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup(world, backend="gloo")
    bench.barrier(w)
    ms = bench.dist_max(100.0 + 10.0 * r, w)  # the slower rank's time wins
    value = bench.job_value(1000, 10, w, ms)
    bench.barrier(w)
    with open(os.path.join(out, "rank%d" % r), "w") as f:
        f.write("%d %d %r %r" % (w, r, ms, value))
    dist.destroy_process_group()


def test_two_gloo_ranks_time_as_the_slowest_and_count_all_replicas(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    for r in range(world):
        w, rr, ms, value = open(tmp_path / ("rank%d" % r)).read().split()
        assert int(w) == world and int(rr) == r
        assert float(ms) == 110.0
        assert abs(float(value) - 1000 * 10 * world / 0.110) < 1e-6
