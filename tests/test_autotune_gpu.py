"""The schedule autotuner (hm_autotune) and the full batching workload.

The autotuner may only change how fast the product runs: the product after
tuning equals the one before up to the order of FP32 sums.  Its choice is
cached per (GPU, matrix shape) in a text file, and a second call with the
same shape applies the cached choice without timing.  The last test runs the
batching workload at its stated size: 64 clouds of 2048-65536 points
(log-uniform, multiples of 32), exp(-r/0.1), tolerance 1e-5, 32 right-hand
sides per cloud, built as one batch, tuned, and multiplied by one graph
launch."""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hm():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hmatrix

    return hmatrix


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_keeps_the_product_and_caches(hm, precision, tmp_path):
    import torch

    n = 1 << 16
    pts = hm.generate_dataset(n, 3, seed=12)
    tree = hm.construct_kdtree(pts, n, 3, 64)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=1e-4, max_rank=128,
                         precision=precision)
    X = torch.randn((n, 16), device="cuda").t().contiguous().t()
    Y0 = H.matvec(X)
    cache = str(tmp_path / "tune.txt")
    choice, cached = hm.autotune(H, 16, cache)
    assert not cached and choice.startswith("mixed" if precision else "fp32")
    Y1 = H.matvec(X)
    assert (torch.linalg.norm(Y1 - Y0) / torch.linalg.norm(Y0)).item() < 1e-6
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1 and ("/mixed/" if precision else "/fp32/") in lines[0]
    choice2, cached2 = hm.autotune(H, 16, cache)
    assert cached2 and choice2 == choice
    assert len(open(cache).read().strip().splitlines()) == 1


def test_batching_workload_full_size(hm, tmp_path):
    import torch

    rng = np.random.default_rng(2024)
    sizes = [int(max(32, round(x / 32) * 32)) for x in np.exp(rng.uniform(np.log(2048), np.log(65536), 64))]
    clouds = []
    for i, n in enumerate(sizes):
        pts = hm.generate_dataset(n, 3, seed=500 + i)
        tree = hm.construct_kdtree(pts, n, 3, 64)
        st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
        clouds.append((n, pts, tree, st))
    B = hm.Batch([c[2] for c in clouds], [c[3] for c in clouds])
    assert B.n == sum(sizes) and B.depth <= 16
    B.build(kernel=hm.K_EXP, ell=0.1, tol=1e-5, max_rank=256, seed=3)
    H = B.hmatrix()
    assert H.stats()["num_unconverged"] == 0
    choice, _ = hm.autotune(H, 16, str(tmp_path / "tune.txt"))
    s = torch.cuda.Stream()
    nrhs = 32
    X = torch.randn((nrhs, B.n), device="cuda").t()
    Y = torch.empty((nrhs, B.n), device="cuda").t()
    with torch.cuda.stream(s):
        B.matvec(X, Y, s)
    s.synchronize()
    Yb = Y.cpu().numpy()
    for c in rng.choice(len(clouds), 6, replace=False):
        n, pts, tree, st = clouds[c]
        r0, r1 = B.row_offsets[c], B.row_offsets[c + 1]
        perm = tree.copy_out()["perm"]
        rows = rng.choice(n, 100, replace=False)
        Xc = X[r0:r1].cpu().numpy().astype(np.float64)
        Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, 3, perm, oracle.K_EXP, 0.1, 0.0, rows, Xc.T).T
        err = np.linalg.norm(Yb[r0:r1][rows] - Yref) / np.linalg.norm(Yref)
        assert err < 20 * 1e-5, (c, n, err)


def test_fp32_panels_match_the_per_block_kernels(hm):
    """The FP32 form has two products: FP32 tiles on the factor panels (the
    default) and the per-block kernels; both are 3xTF32, so they agree to FP32
    rounding, in tree and in original order and over several passes."""
    import torch

    n = 1 << 16
    pts = hm.generate_dataset(n, 3, seed=21)
    tree = hm.construct_kdtree(pts, n, 3, 64)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.2, tol=1e-6, max_rank=128)
    X = torch.randn((n, 37), device="cuda").t().contiguous().t()
    for order in (False, True):
        hm.schedule_set(H, "fp32 chunk_tiles=32 group_tiles=4")
        Yp = H.matvec(X, original_order=order)
        hm.schedule_set(H, "fp32 p1_rows=512")
        Yb = H.matvec(X, original_order=order)
        rel = (torch.linalg.norm(Yp - Yb) / torch.linalg.norm(Yb)).item()
        assert rel < 1e-6, (order, rel)
    perm = tree.copy_out()["perm"]
    rows = np.random.default_rng(3).choice(n, 128, replace=False)
    hm.schedule_set(H, "fp32 chunk_tiles=128 group_tiles=2")
    Y = H.matvec(X[:, :5]).cpu().numpy()
    Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, 3, perm, oracle.K_EXP, 0.2, 0.0, rows,
                                    X[:, :5].t().cpu().numpy().astype(np.float64)).T
    assert np.linalg.norm(Y[rows] - Yref) / np.linalg.norm(Yref) < 5e-6
