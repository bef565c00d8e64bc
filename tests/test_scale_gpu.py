"""Scale-stress form: points from a 16-component isotropic Gaussian mixture
(centres uniform in [0,1]^3, sigma log-uniform in [0.01, 0.1], Dirichlet(1)
weights), so the KD tree splits unevenly and ranks vary; exp(-r/0.05),
box-center eta = 1.5, tolerance 1e-4, rank cap 256, 128 right-hand sides.

With eta = 1.5 some admissible blocks need more than 256 columns; such a
block is compressed as its four child blocks instead (num_split), so every
stored block meets the tolerance (num_unconverged == 0).  Checked at 2^17
points (both forms) and at the full 2^21 points (mixed form): the product
against the FP64 oracle on seeded rows, and sampled blocks against the
oracle's per-block error ||A - U V^T||_F / ||A||_F <= tol."""
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


def test_mixture_generator_is_seeded(hm):
    a = hm.generate_mixture(5000, 3, seed=9).cpu().numpy()
    b = hm.generate_mixture(5000, 3, seed=9).cpu().numpy()
    c = hm.generate_mixture(5000, 3, seed=10).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    x = a.reshape(3, 5000)
    assert np.isfinite(x).all()
    # clustered: a uniform cloud of 5000 points leaves about 1% of a 10^3 grid
    # over [0,1]^3 empty; 16 components with sigma <= 0.1 leave far more
    inside = np.all((x >= 0) & (x < 1), axis=0)
    cells = np.unique((np.floor(x[:, inside] * 10)).astype(int), axis=1).shape[1]
    assert cells < 0.8 * 1000, cells


def _block_errors(hm, H, ph, n, d, perm, tol, nsample, max_entries, seed):
    """Per-block errors of up to nsample low-rank blocks (of at most
    max_entries entries), the largest levels first, against the FP64 oracle."""
    lr, _ = H.blocks()
    rng = np.random.default_rng(seed)
    ok = np.nonzero(lr[:, 1].astype(np.int64) * lr[:, 3] <= max_entries)[0]
    levels = np.unique(lr[ok, 5])
    pick = []
    for lv in levels:  # every level present, then random others
        cand = ok[lr[ok, 5] == lv]
        pick.append(int(rng.choice(cand)))
    rest = np.setdiff1d(ok, pick)
    pick += [int(i) for i in rng.choice(rest, min(len(rest), max(0, nsample - len(pick))), replace=False)]
    errs = []
    for i in pick:
        r0, m, c0, nc, k, lvl = (int(x) for x in lr[i])
        U, V = H.block_factors(i)
        errs.append(oracle.block_error(ph, n, d, perm, oracle.K_EXP, 0.05, 0.0, r0, m, c0, nc, U, V))
    return np.array(errs)


def test_scale_stress_reduced(hm):
    import torch

    n, d, b = 1 << 17, 3, 64
    pts = hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=77)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.5)
    perm = tree.copy_out()["perm"]
    ph = pts.cpu().numpy()
    X = torch.randn((128, n), device="cuda").t()
    rng = np.random.default_rng(1)
    rows = rng.choice(n, 1024, replace=False)
    Yref = oracle.dense_rows_matvec(ph, n, d, perm, oracle.K_EXP, 0.05, 0.0, rows,
                                    X.t().cpu().numpy().astype(np.float64)).T
    for prec in (hm.PREC_FP32, hm.PREC_MIXED):
        H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.05, tol=1e-4, max_rank=256, precision=prec,
                             seed=5)
        s = H.stats()
        assert s["num_unconverged"] == 0, s
        Y = H.matvec(X).cpu().numpy()
        err = np.linalg.norm(Y[rows] - Yref) / np.linalg.norm(Yref)
        assert err < 1e-4, (prec, err, s)
        e = _block_errors(hm, H, ph, n, d, perm, 1e-4, 24, 1 << 22, 3)
        assert e.max() <= 1e-4, (prec, e)


def test_scale_stress_full_size(hm):
    """The scale-stress workload at its full size: 2^21 mixture points, 128
    right-hand sides, mixed precision.  Error on 4096 seeded rows in the first
    and the last 16 columns (one from each 64-column pass of the product)."""
    import torch

    n, d, b = 1 << 21, 3, 64
    pts = hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=1234)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.5)
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.05, tol=1e-4, max_rank=256,
                         precision=hm.PREC_MIXED, seed=7)
    s = H.stats()
    assert s["num_unconverged"] == 0, s
    assert s["max_rank_seen"] <= 256, s
    gen = torch.Generator(device="cuda")
    gen.manual_seed(99)
    X = torch.randn((128, n), generator=gen, device="cuda").t()
    Y = H.matvec(X).cpu().numpy()
    perm = tree.copy_out()["perm"]
    ph = pts.cpu().numpy()
    rows = np.random.default_rng(5).choice(n, 4096, replace=False)
    cols = np.r_[0:16, 112:128]
    Xc = X.t().cpu().numpy()[cols].astype(np.float64)
    Yref = oracle.dense_rows_matvec(ph, n, d, perm, oracle.K_EXP, 0.05, 0.0, rows, Xc).T
    err = np.linalg.norm(Y[rows][:, cols] - Yref) / np.linalg.norm(Yref)
    assert err <= 1e-4, (err, s)
    e = _block_errors(hm, H, ph, n, d, perm, 1e-4, 16, 1 << 22, 11)
    assert e.max() <= 1e-4, e
