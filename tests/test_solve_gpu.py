"""Conjugate gradients on the H-matrix (hm_cg_solve): a kernel with a nugget
on its diagonal is symmetric positive definite, and CG solves H X = B with
the H-matrix product as its operator.  The solution is checked against a
dense FP64 solve of the same kernel matrix built by the oracle
(src/expandMatrix.cu:142-231 restated), the reported residual against a
residual recomputed here, and the graph-launched chunks (created stream)
against direct launches (legacy stream)."""
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


N, D, B = 4096, 3, 64
ELL, NUGGET = 0.2, 1.0


@pytest.fixture(scope="module")
def cloud(hm):
    pts = hm.generate_dataset(N, D, seed=77)
    tree = hm.construct_kdtree(pts, N, D, B)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    perm = tree.copy_out()["perm"]
    p_h = pts.cpu().numpy()
    A = oracle.dense_block(p_h, N, D, perm, oracle.K_MATERN32, ELL, NUGGET, 0, N, 0, N)  # tree order, FP64
    return pts, tree, st, A


# (the mixed form's product rounds X and, for columns without low parts, the
# projections to BF16, so it is linear only to about 1e-4: its true residual
# levels off there while CG's recurrence keeps shrinking)
@pytest.mark.parametrize("precision,tol_build,tol_cg,res_bound,bound",
                         [(0, 1e-6, 1e-6, 5e-6, 2e-3), (1, 1e-4, 1e-5, 2e-4, 5e-2)])
def test_cg_matches_dense_solve(hm, cloud, precision, tol_build, tol_cg, res_bound, bound):
    import torch

    pts, tree, st, A = cloud
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=ELL, nugget=NUGGET, tol=tol_build, max_rank=64,
                         precision=precision)
    rng = np.random.default_rng(3)
    Bn = rng.standard_normal((N, 4))
    Bt = torch.from_numpy(Bn.astype(np.float32)).cuda()
    X, iters, res = hm.cg_solve(H, Bt, tol=tol_cg, max_iter=2000)
    assert 0 < iters <= 2000
    # the reported residual is the true one, ||B - H X|| / ||B|| per column
    R = (Bt - H.matvec(X)).cpu().numpy()
    mine = max(np.linalg.norm(R[:, j]) / np.linalg.norm(Bn[:, j]) for j in range(4))
    assert abs(mine - res) <= 1e-6 + 0.05 * res, (mine, res)
    assert res <= res_bound, res
    # against the dense FP64 solve of the kernel matrix
    Xref = np.linalg.solve(A, Bn)
    err = np.linalg.norm(X.cpu().numpy() - Xref) / np.linalg.norm(Xref)
    assert err < bound, err


def test_cg_graph_chunks_equal_direct_launches(hm, cloud):
    """A created stream runs each chunk of iterations as a recorded graph; the
    legacy stream launches the same kernels directly.  Same iterates; a zero
    right-hand side stays zero."""
    import torch

    pts, tree, st, A = cloud
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=ELL, nugget=NUGGET, tol=1e-6, max_rank=64)
    Bt = torch.randn((3, N), device="cuda").t()  # (N, 3), columns contiguous
    Bt[:, 1] = 0
    X0, it0, r0 = hm.cg_solve(H, Bt, tol=1e-6, max_iter=500, check_every=8)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        X1, it1, r1 = hm.cg_solve(H, Bt, tol=1e-6, max_iter=500, check_every=8, stream=s)
    s.synchronize()
    assert it0 == it1
    torch.testing.assert_close(X1, X0, rtol=0, atol=0)
    assert torch.count_nonzero(X0[:, 1]).item() == 0


def test_cg_reports_non_convergence_and_indefinite(hm, cloud):
    import torch

    pts, tree, st, A = cloud
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=ELL, nugget=NUGGET, tol=1e-6, max_rank=64)
    Bt = torch.randn((N, 2), device="cuda")
    with pytest.raises(hm.HMError) as e:
        hm.cg_solve(H, Bt, tol=1e-12, max_iter=3, check_every=2)
    assert e.value.status == 6
    # a negative nugget larger than the average eigenvalue makes p.Ap < 0 at once
    Hn = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=ELL, nugget=-10.0, tol=1e-6, max_rank=64)
    with pytest.raises(hm.HMError) as e:
        hm.cg_solve(Hn, Bt, tol=1e-6, max_iter=50)
    assert e.value.status == 4
    with pytest.raises(hm.HMError):
        hm.cg_solve(H, Bt, tol=0.0)
