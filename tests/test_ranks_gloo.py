"""The benchmark's multi-rank logic on CPU: two gloo ranks on 127.0.0.1."""
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "kaust-hierarchical-matrices_b200")


def _worker(rank, world, port, q):
    sys.path.insert(0, PKG)
    import datetime

    import torch.distributed as dist

    import ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = ranks.max_over_ranks(1.5 + rank, world)  # the slowest rank sets the step time
        v = ranks.weak_value(3e9, ms, world)
        q.put((rank, ms, v, ranks.cloud_seed(1234, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [2.5, 2.5]                 # max over ranks on both
    assert all(abs(o[2] - 2 * 3e9 / 2.5e-3 / 1e9) < 1e-9 for o in out)
    assert out[0][3] != out[1][3]                            # independent clouds


def test_single_rank_is_identity():
    sys.path.insert(0, PKG)
    import ranks

    assert ranks.max_over_ranks(3.25, 1) == 3.25
    assert ranks.weak_value(1e9, 1.0, 1) == pytest.approx(1000.0)
