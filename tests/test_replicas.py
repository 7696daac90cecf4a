"""The N-GPU bench path on the CPU: replicas only (no data-path collective),
timed as the maximum over ranks. Two gloo ranks on 127.0.0.1 run the bench's
own helpers; the reference arm runs on rank 0 alone."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import argparse
    import datetime

    import torch.distributed as dist

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench._dist()
        slowest = bench._max_over_ranks(10.0 + 5.0 * rank, w, "cpu")
        # The reference arm: a rank other than 0 returns at once, without work.
        reference = bench.run_reference(argparse.Namespace(size=96, seed=1), r, w) if r else "rank0"
        out.put((r, w, local, slowest, reference))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_report_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=100) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r[:3] for r in results] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == 15.0 for r in results)  # both ranks see the slowest
    assert results[1][4] is None  # the reference arm: rank 0 alone runs it


def test_single_rank_time_is_unchanged():
    import bench
    assert bench._max_over_ranks(12.5, 1, "cpu") == 12.5
