"""The bench's multi-process path on the CPU: two gloo ranks (one process each, as under
torchrun) agree on the slowest rank's time and on the whole-job throughput, and draw
different ray batches.  No GPU: replicas have no data-path collective, so this is all the
N>1 path does besides running the single-GPU step on each rank."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import sys
    from datetime import timedelta

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench

    torch.distributed.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        got_ws, got_rank, _ = bench.dist_env()
        times = bench.max_over_ranks([10.0 + rank, 5.0 * (1 + rank), 1.0], "cpu", got_ws)
        value = bench.job_throughput(65536, 4, got_ws, times[0])
        gen = torch.Generator().manual_seed(1000 + got_rank)  # the seed of each rank's batches in bench.py
        draw = torch.randint(0, 1 << 20, (8,), generator=gen).tolist()
        out.put((got_rank, times, value, draw))
    finally:
        torch.distributed.destroy_process_group()


def test_two_rank_timing_and_throughput():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, d0), (r1, t1, v1, d1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == [11.0, 10.0, 1.0]  # each entry is the maximum over the ranks
    assert v0 == v1 == pytest.approx(65536 * 4 * 2 / 0.011)
    assert d0 != d1
