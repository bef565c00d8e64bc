"""Block-row shards of one cloud (hm_hmatrix_build_rows) on one GPU.

The ranks of a multi-GPU product are emulated one after another on one GPU:
each shard is built from the same tree and structure, multiplies the whole X
and contributes its own rows.  Stacked, the shards' rows must give the whole
matrix's product (the same blocks per row, in the same order), and each shard
holds fewer blocks than the whole matrix.  Also checks hm_hmatvec_f64 (the
reference's FP64 vectors) against hm_hmatvec.
"""
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


@pytest.fixture(scope="module")
def cloud(hm):
    n, d, b = 1 << 16, 3, 64
    pts = hm.generate_dataset(n, d, seed=31)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    return n, d, pts, tree, st


@pytest.mark.parametrize("prec", [0, 1])
def test_row_shards_stack_to_the_product(hm, cloud, prec):
    import torch

    import ranks

    n, d, pts, tree, st = cloud
    kw = dict(kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=1e-5, max_rank=128, precision=prec, seed=3)
    H = hm.build_hmatrix(tree, st, pts, **kw)
    X = torch.randn((20, n), device="cuda").t()
    Yfull = H.matvec(X)
    full_blocks = H.stats()["num_lowrank"]
    offs = tree.copy_out()["offsets"]
    for world in (2, 3):
        Y = torch.full_like(Yfull, float("nan"))
        for lb, le, r0, r1 in ranks.subtree_shards(list(offs), world):
            Hs = hm.build_hmatrix(tree, st, pts, leaves=(lb, le), **kw)
            assert Hs.stats()["num_lowrank"] < full_blocks
            Yr = torch.full_like(Yfull, float("nan"))
            Hs.matvec(X, Y=Yr)
            assert torch.isnan(Yr[:r0]).all() and torch.isnan(Yr[r1:]).all()  # other rows untouched
            Y[r0:r1] = Yr[r0:r1]
            del Hs
        rel = (torch.linalg.norm(Y - Yfull) / torch.linalg.norm(Yfull)).item()
        assert rel < 1e-6, (world, rel)


def test_fp64_vectors_match_fp32_product(hm, cloud):
    import torch

    n, d, pts, tree, st = cloud
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.2, tol=1e-6, max_rank=128, seed=4)
    X = torch.randn((5, n), device="cuda", dtype=torch.float64).t()
    Y64 = H.matvec_f64(X)
    Y32 = H.matvec(X.float())
    assert Y64.dtype == torch.float64
    assert torch.equal(Y64.float(), Y32)  # same FP32 product, widened
    # original order: the permutation applied by the conversion kernels
    Yo = H.matvec_f64(X, original_order=True)
    Yo32 = H.matvec(X.float(), original_order=True)
    assert torch.equal(Yo.float(), Yo32)
    # and against the FP64 oracle on sampled rows (tree order)
    perm = tree.copy_out()["perm"]
    rows = np.random.default_rng(2).choice(n, 200, replace=False)
    Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, d, perm, oracle.K_EXP, 0.2, 0.0, rows,
                                    X.t().cpu().numpy()).T
    err = np.linalg.norm(Y64.cpu().numpy()[rows] - Yref) / np.linalg.norm(Yref)
    assert err < 1e-5, err


@pytest.mark.parametrize("prec", [0, 1])
def test_piecewise_out_of_core_product(hm, cloud, prec, tmp_path):
    """The out-of-core form: the matrix built as three block-row pieces, each
    written to a file and freed; the product loads one piece at a time.  It
    equals the in-memory product, and no piece needs the whole matrix's
    device memory."""
    import torch

    n, d, pts, tree, st = cloud
    kw = dict(kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=1e-5, max_rank=128, precision=prec, seed=3)
    H = hm.build_hmatrix(tree, st, pts, **kw)
    X = torch.randn((7, n), device="cuda").t()
    Y = H.matvec(X)
    whole = H.stats()["device_bytes"]
    del H
    P = hm.PiecewiseHMatrix(tree, st, pts, 3, tmp_path, **kw)
    assert max(P.piece_device_bytes) < whole
    Yp = P.matvec(X)
    rel = (torch.linalg.norm(Yp - Y) / torch.linalg.norm(Y)).item()
    assert rel < 1e-6, rel
