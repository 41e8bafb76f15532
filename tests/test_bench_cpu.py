"""The bench's multi-rank logic on CPU: two gloo ranks (world size 2, as
torchrun launches them) take the slowest rank's time, and the reference arm
runs on rank 0 only."""
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
        env = bench.dist_env()
        # the reference arm: ranks other than 0 return at once and print nothing
        ref = bench.run_reference(None, rank, world) if rank != 0 else None
        dist.barrier()
        q.put((rank, got, env, ref))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 15.0 for r in res)            # the slower rank's time on both
    assert [r[2] for r in res] == [(0, 0, 2), (1, 1, 2)]
    assert res[1][3] is None
    assert all(p.exitcode == 0 for p in procs)


def test_max_over_ranks_without_a_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, "cpu") == 3.25
