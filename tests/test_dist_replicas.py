"""Multi-GPU plumbing of bench.py on CPU: two gloo ranks.

The path runs as replicas: each rank proves its own copy of the workload and
the only collectives are the barrier around the timed region and one
all-reduce of the timing scalar (max over ranks).  This runs those helpers in
two spawned processes over gloo and checks that both ranks see the slowest
rank's time and the whole-job (weak-scaling) rate.
"""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    os.environ.update(WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    bench.dist_backend = lambda: "gloo"  # CPU ranks, whatever the host has
    world, r, _ = bench.dist_setup()
    bench.barrier(world)
    ms = bench.max_over_ranks(2.0 + 3.0 * rank, world)  # rank 1 is the slower one
    q.put((r, world, ms, bench.replica_rate(1000.0, ms, world)))
    bench.barrier(world)
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    for r, (rank, world, ms, rate) in enumerate(got):
        assert rank == r and world == 2
        assert ms == 5.0  # max over ranks
        assert abs(rate - 2 * 1000.0 / 5e-3) < 1e-6  # 2 replicas of 1000 units in 5 ms


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.replica_rate(10.0, 2.0, 1) == 5000.0
