"""The mixed form's 128-column passes on tcgen05 (hm_mixed_tc.cu).

With wide_tc=1 in the schedule, a pass of 65-128 right-hand sides runs both
phases with tcgen05.mma (accumulator in tensor memory); wide_tc=0 (the
default) runs the warp-level MMA kernels.  Both compute the same sums (up to the
order of FP32 additions), so their products agree to FP32 rounding; both
agree with the same columns multiplied 16 at a time, and with the FP64
oracle on sampled rows at the build tolerance.  Cases cover panels projected
in one row chunk (T stored by phase 1) and in several (chunk partials,
remainder chunks), units with and without low parts, an odd number of row
tiles per unit, leaves of one and of two row tiles (phase-2 blocks of 4 row
tiles that span 2 or 4 leaves), and a pass narrower than 128 columns.
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


CASES = [
    # n, d, b, chunk tiles (None: default schedule), right-hand sides
    (1 << 16, 3, 64, None, 128),
    (50000, 2, 32, 48, 100),
    (24000, 3, 64, 16, 77),
]


@pytest.mark.parametrize("n,d,b,chunk,nrhs", CASES)
def test_tc_phase1_matches_warp_phase1(hm, n, d, b, chunk, nrhs):
    import torch

    kind, ell, nugget, tol = hm.K_MATERN32, 0.2, 1e-3, 1e-4
    pts = hm.generate_dataset(n, d, seed=5)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    H = hm.build_hmatrix(tree, st, pts, kernel=kind, ell=ell, nugget=nugget, tol=tol, max_rank=128,
                         precision=hm.PREC_MIXED)
    ch = 128 if chunk is None else chunk
    X = torch.randn((nrhs, n), device="cuda", dtype=torch.float32).t()
    hm.schedule_set(H, f"mixed chunk_tiles={ch} group_tiles=4 p1_ring=0 wide_tc=1")
    Ytc = H.matvec(X)
    H.check()
    hm.schedule_set(H, f"mixed chunk_tiles={ch} group_tiles=4 p1_ring=0 wide_tc=0")
    Yw = H.matvec(X)
    parts = torch.cat([H.matvec(X[:, c0:min(c0 + 16, nrhs)].t().contiguous().t()) for c0 in range(0, nrhs, 16)],
                      dim=1)
    scale = torch.linalg.norm(Yw).item()
    assert torch.isfinite(Ytc).all()
    d_tc = torch.linalg.norm(Ytc - Yw).item() / scale
    d_parts = torch.linalg.norm(Ytc - parts).item() / scale
    assert d_tc <= 2e-6, d_tc
    assert d_parts <= 2e-6, d_parts
    # against the FP64 oracle on sampled rows (tree order), a few columns
    perm = tree.copy_out()["perm"]
    rows = np.random.default_rng(3).choice(n, 256, replace=False)
    cols = [0, nrhs // 2, nrhs - 1]
    Xc = X[:, cols].t().cpu().numpy().astype(np.float64)
    Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, d, perm, oracle.K_MATERN32, ell, nugget, rows, Xc).T
    err = np.linalg.norm(Ytc[:, cols].cpu().numpy()[rows] - Yref) / np.linalg.norm(Yref)
    assert err < 1e-4, err


def test_tc_phase1_repeats_bit_for_bit(hm):
    """The tcgen05 pass is deterministic: fixed unit order per CTA, fixed MMA
    chains, and the chunk partials summed in chunk order."""
    import torch

    n = 1 << 15
    pts = hm.generate_dataset(n, 3, seed=8)
    tree = hm.construct_kdtree(pts, n, 3, 64)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.2, tol=1e-5, max_rank=128, precision=hm.PREC_MIXED)
    X = torch.randn((128, n), device="cuda", dtype=torch.float32).t()
    hm.schedule_set(H, "mixed chunk_tiles=128 group_tiles=4 p1_ring=0 wide_tc=1")
    Y1 = H.matvec(X)
    Y2 = H.matvec(X)
    H.check()
    assert torch.equal(Y1, Y2)
