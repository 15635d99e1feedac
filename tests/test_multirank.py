"""Replica (N > 1) plumbing of bench.py on CPU: two gloo ranks.

Clips are independent, so N GPUs run N replicas with no collective on the
data path; the only collectives are the barrier and the max over ranks of
the timed region.  These tests run that logic as two processes on the CPU.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        ms = bench.max_over_ranks(times[rank], world)
        value = bench.whole_job_rate(world, bench.N_CLIPS, ms)
        bench.barrier(world)
        q.put((rank, ms, value, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_disjoint_clips():
    import bench
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    times = [12.5, 20.0]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the max over ranks; the rate counts both ranks' clips
    assert [o[1] for o in out] == [20.0, 20.0]
    assert out[0][2] == pytest.approx(2 * bench.N_CLIPS / 0.020)
    # replicas draw disjoint seed ranges of N_CLIPS clips each
    s0, s1 = out[0][3], out[1][3]
    assert abs(s1 - s0) >= bench.N_CLIPS


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.whole_job_rate(1, 256, 5.0) == pytest.approx(256 / 0.005)
