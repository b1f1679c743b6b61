"""The multi-rank path of bench.py on CPU: two gloo ranks over 127.0.0.1 take the same collective steps as
the timed region (barrier, max of the step times, sum of the converged counts), and the reference arm runs on
rank 0 alone while the other rank exits without work."""

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


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist()
    try:
        d.barrier()
        ms_max = d.reduce([1.0 + rank], "max")[0]  # per-rank step time: the job takes the slowest
        conv, probs = d.reduce([10.0 * (rank + 1), 100.0], "sum")
        ref = bench.run_reference(None, d) if rank == 1 else None  # rank 1 of the reference arm: no work
        out.put((rank, ms_max, conv, probs, ref))
    finally:
        d.close()


def test_two_gloo_ranks_reduce_like_the_timed_region():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms_max, conv, probs, ref in res:
        assert ms_max == 2.0 and conv == 30.0 and probs == 200.0
    assert res[1][4] == {}


@pytest.mark.parametrize("world", [1])
def test_single_rank_needs_no_process_group(world):
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist()
    assert d.world == 1 and d.reduce([3.0], "max") == [3.0]
    d.barrier()
    d.close()
