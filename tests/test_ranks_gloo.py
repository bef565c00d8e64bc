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


def test_cloud_assignment_is_balanced():
    sys.path.insert(0, PKG)
    import numpy as np

    import ranks

    rng = np.random.default_rng(2024)
    sizes = [int(round(x / 32) * 32) for x in np.exp(rng.uniform(np.log(2048), np.log(65536), 64))]
    for world in (1, 2, 3, 4, 8):
        parts = ranks.assign_clouds(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(64))  # each cloud exactly once
        loads = [sum(ranks.cloud_cost(sizes[i]) for i in p) for p in parts]
        # longest-first greedy: within one cloud of the mean
        assert max(loads) - min(loads) <= max(ranks.cloud_cost(s) for s in sizes) + 1e-6
        assert all(len(p) >= 1 for p in parts)


def test_subtree_shards_cover_the_rows():
    sys.path.insert(0, PKG)
    import oracle
    import ranks

    for n, b in ((1 << 20, 64), (50016, 64), (8192, 32)):
        depth = oracle.tree_depth(n, b)
        # the FULL_TREE leaf offsets (ceil halvings), as hm_kdtree_build makes them
        offs = [0, n]
        for _ in range(depth):
            nx = [0]
            for s in range(len(offs) - 1):
                ln = offs[s + 1] - offs[s]
                nx += [offs[s] + (ln + 1) // 2, offs[s + 1]]
            offs = nx
        for world in (1, 2, 3, 4, 5, 8):
            sh = ranks.subtree_shards(offs, world)
            assert len(sh) == world
            assert sh[0][0] == 0 and sh[-1][1] == 1 << depth and sh[0][2] == 0 and sh[-1][3] == n
            L = (world - 1).bit_length()
            per = (1 << depth) >> L
            for a, b_ in zip(sh, sh[1:]):
                assert a[1] == b_[0] and a[3] == b_[2]    # contiguous
            for lb, le, r0, r1 in sh:
                assert lb % per == 0 and le % per == 0 and le > lb  # whole subtrees of level L
                assert offs[lb] == r0 and offs[le] == r1
            rows = [r1 - r0 for *_, r0, r1 in sh]
            assert max(rows) <= 2 * n / world + 1              # near an equal share


def _shard_worker(rank, world, port, q):
    """One cloud split by block rows: X's rows spread over the ranks are
    all-gathered, each rank multiplies its own rows (a CPU stand-in for the
    device product: the oracle's dense FP64 rows), and the rows are gathered
    back into the whole Y."""
    sys.path.insert(0, PKG)
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import oracle
    import ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n, d, b, nrhs = 3000, 2, 32, 3
        rng = np.random.default_rng(7)  # the same cloud and X on every rank
        pts = rng.uniform(size=d * n)
        X = rng.standard_normal((nrhs, n))
        t = oracle.kdtree(pts, n, d, b)
        shards = ranks.subtree_shards(list(t["offsets"]), world)
        _, _, r0, r1 = shards[rank]
        x_local = torch.from_numpy(np.ascontiguousarray(X[:, r0:r1]))
        x_full = ranks.allgather_rows(x_local, shards, rank).numpy()
        y_local = oracle.dense_rows_matvec(pts, n, d, t["perm"], oracle.K_EXP, 0.1, 0.0, np.arange(r0, r1), x_full)
        y_full = ranks.allgather_rows(torch.from_numpy(np.ascontiguousarray(y_local)), shards, rank).numpy()
        y_ref = oracle.dense_rows_matvec(pts, n, d, t["perm"], oracle.K_EXP, 0.1, 0.0, np.arange(n), X)
        q.put((rank, bool(np.array_equal(x_full, X)), float(np.abs(y_full - y_ref).max())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_row_shards_assemble_the_product(world):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert all(o[1] for o in out)      # X gathered exactly
    assert all(o[2] == 0.0 for o in out)  # each row computed once, by its owner, in the same order
