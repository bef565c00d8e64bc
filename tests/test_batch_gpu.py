"""Batching form through the C ABI: independent clouds of uneven size joined
as one forest (hm_batch_*), built together, multiplied by one CUDA-graph
launch over all clouds.  Each cloud's rows of the batched product are checked
against the FP64 oracle on that cloud alone (src/expandMatrix.cu:142-231), and
against the cloud built and multiplied on its own."""
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


def cloud_sizes(count, lo, hi, seed):
    """Sizes drawn log-uniform in [lo, hi], rounded to a multiple of 32."""
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), count))
    return [int(max(32, round(x / 32) * 32)) for x in s]


def make_clouds(hm, sizes, d=3, b=64, seed0=100):
    clouds = []
    for i, n in enumerate(sizes):
        pts = hm.generate_dataset(n, d, seed=seed0 + i)
        tree = hm.construct_kdtree(pts, n, d, b)
        st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
        clouds.append((n, pts, tree, st))
    return clouds


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_product_matches_oracle_and_single_clouds(hm, precision):
    import torch

    kind, ell, tol, nrhs = hm.K_EXP, 0.1, 1e-5, 32
    sizes = cloud_sizes(9, 2048, 16384, seed=3)
    clouds = make_clouds(hm, sizes)
    B = hm.Batch([c[2] for c in clouds], [c[3] for c in clouds])
    assert B.nclouds == 9 and B.n == sum(sizes) and B.row_offsets[-1] == B.n
    B.build(kernel=kind, ell=ell, tol=tol, max_rank=64, precision=precision, seed=1)
    s = torch.cuda.Stream()
    X = torch.randn((B.n, nrhs), device="cuda").t().contiguous().t()  # column-major
    Y = torch.empty((nrhs, B.n), device="cuda").t()
    with torch.cuda.stream(s):
        B.matvec(X, Y, s)
        B.matvec(X, Y, s)  # relaunch of the recorded graph
    s.synchronize()
    Yb = Y.cpu().numpy()
    rng = np.random.default_rng(0)
    for c, (n, pts, tree, st) in enumerate(clouds):
        r0, r1 = B.row_offsets[c], B.row_offsets[c + 1]
        Xc = X[r0:r1].cpu().numpy().astype(np.float64)
        perm = tree.copy_out()["perm"]
        rows = rng.choice(n, min(n, 200), replace=False)
        Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, 3, perm, kind, ell, 0.0, rows, Xc.T).T
        err = np.linalg.norm(Yb[r0:r1][rows] - Yref) / np.linalg.norm(Yref)
        assert err < 20 * tol, (c, n, err)
        if c < 3:  # the same cloud on its own
            H = hm.build_hmatrix(tree, st, pts, kernel=kind, ell=ell, tol=tol, max_rank=64, precision=precision,
                                 seed=1)
            Ys = H.matvec(X[r0:r1].contiguous().t().contiguous().t()).cpu().numpy()
            assert np.linalg.norm(Ys - Yb[r0:r1]) <= 20 * tol * np.linalg.norm(Ys)


def test_batch_graph_follows_data_and_arguments(hm):
    """The recorded graph reads the buffers' current contents; a call with
    other arguments records a new graph; original order maps each cloud's rows
    through its own permutation."""
    import torch

    sizes = [4096, 2080, 7200]
    clouds = make_clouds(hm, sizes, seed0=40)
    B = hm.Batch([c[2] for c in clouds], [c[3] for c in clouds])
    B.build(kernel=hm.K_EXP, ell=0.1, tol=1e-5, max_rank=64)
    H = B.hmatrix()
    s = torch.cuda.Stream()
    X = torch.empty((5, B.n), device="cuda").t()
    Y = torch.empty((5, B.n), device="cuda").t()
    with torch.cuda.stream(s):
        for trial in range(2):
            X.copy_(torch.randn((B.n, 5), device="cuda"))
            B.matvec(X, Y, s)
            s.synchronize()
            Yd = H.matvec(X.contiguous().t().contiguous().t(), stream=s)
            s.synchronize()
            torch.testing.assert_close(Y, Yd, rtol=0, atol=0)
        # other width: a new graph
        X3, Y3 = X[:, :3].contiguous().t().contiguous().t(), torch.empty((3, B.n), device="cuda").t()
        B.matvec(X3, Y3, s)
        s.synchronize()
        torch.testing.assert_close(Y3, Y[:, :3], rtol=0, atol=0)
        # original order: cloud c's original point i is row row_offsets[c] + i
        perms = [c[2].copy_out()["perm"] for c in clouds]
        gperm = np.concatenate([p + B.row_offsets[c] for c, p in enumerate(perms)])
        Xo = torch.empty_like(X)
        Xo[torch.from_numpy(gperm).cuda().long()] = X
        Yo = torch.empty_like(Y)
        B.matvec(Xo, Yo, s, original_order=True)
        s.synchronize()
    torch.testing.assert_close(Yo[torch.from_numpy(gperm).cuda().long()], Y, rtol=1e-6, atol=1e-6)


def test_batch_rejects_bad_input(hm):
    import torch

    clouds = make_clouds(hm, [2048, 3000], seed0=70)
    with pytest.raises(hm.HMError):
        hm.Batch([clouds[0][2], clouds[1][2]], [clouds[1][3], clouds[0][3]])  # structure of another tree
    B = hm.Batch([c[2] for c in clouds], [c[3] for c in clouds])
    X = torch.zeros((B.n, 1), device="cuda")
    with pytest.raises(hm.HMError):
        B.matvec(X, X.clone(), torch.cuda.Stream())  # not built
