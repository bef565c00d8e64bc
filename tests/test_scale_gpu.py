"""Scale-stress form at reduced size: points from a 16-component isotropic
Gaussian mixture (centres uniform in [0,1]^3, sigma log-uniform in
[0.01, 0.1], Dirichlet(1) weights), so the KD tree splits unevenly and ranks
vary; exp(-r/0.05), box-center eta = 1.5, tolerance 1e-4, rank cap 256, 128
right-hand sides (eight 16-column panels), mixed precision against the FP32
form.  Both products are checked against the FP64 oracle on sampled rows.""" 
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
    rows = rng.choice(n, 300, replace=False)
    Yref = oracle.dense_rows_matvec(ph, n, d, perm, oracle.K_EXP, 0.05, 0.0, rows,
                                    X.t().cpu().numpy().astype(np.float64)).T
    for prec in (hm.PREC_FP32, hm.PREC_MIXED):
        H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.05, tol=1e-4, max_rank=256, precision=prec,
                             seed=5)
        s = H.stats()
        # with eta = 1.5 a few large blocks need more than the rank cap of 256;
        # they keep their capped factors (counted, not hidden), and the product
        # still meets the bound below
        assert s["num_unconverged"] < 0.001 * s["num_lowrank"], s
        Y = H.matvec(X).cpu().numpy()
        err = np.linalg.norm(Y[rows] - Yref) / np.linalg.norm(Yref)
        assert err < 2e-4, (prec, err, s)
