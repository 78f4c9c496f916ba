"""
Replicas-only multi-rank timing (bench.py): two gloo ranks on CPU check that
the job time is the maximum over ranks and the step count the sum, the two
reductions the benchmark applies to its per-rank CUDA-event timings.
"""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, dist = bench._dist()
    try:
        assert (r, w) == (rank, world) and dist.get_backend() == "gloo"
        t = bench.max_over_ranks(1.0 + 2.5 * rank, dist)        # per-rank seconds
        n = bench.sum_over_ranks(10.0 * (rank + 1), dist)       # per-rank steps
        out.put((rank, t, n))
    finally:
        dist.destroy_process_group()


def test_max_and_sum_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, t, n in got:
        assert t == pytest.approx(3.5)
        assert n == pytest.approx(30.0)
