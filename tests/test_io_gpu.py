"""Binary H-matrix files (hm_hmatrix_save / hm_hmatrix_load): a matrix read
back onto the same tree and structure multiplies exactly like the one that
was saved (same factors, same plans), for the FP32 form, the mixed form and
a derivative build; a file is refused for another cloud, when truncated, or
when it is not an H-matrix file."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hm():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hmatrix

    return hmatrix


def cloud(hm, n, seed):
    pts = hm.generate_dataset(n, 3, seed=seed)
    tree = hm.construct_kdtree(pts, n, 3, 64)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    return pts, tree, st


@pytest.mark.parametrize("precision,derivative", [(0, 0), (1, 0), (0, 1)])
def test_saved_matrix_multiplies_like_the_original(hm, tmp_path, precision, derivative):
    import torch

    n = 20000
    pts, tree, st = cloud(hm, n, 5)
    kind = hm.K_GAUSS if derivative else hm.K_MATERN32
    H = hm.build_hmatrix(tree, st, pts, kernel=kind, ell=0.2, nugget=0.0 if derivative else 1e-3, tol=1e-5,
                         max_rank=64, precision=precision, derivative=derivative)
    path = tmp_path / "h.bin"
    H.save(path)
    H2 = hm.load_hmatrix(tree, st, path)
    s1, s2 = H.stats(), H2.stats()
    for k in ("num_lowrank", "num_dense", "rank_sum", "max_rank_seen", "factor_bytes", "mixed_bytes"):
        assert s1[k] == s2[k], k
    X = torch.randn((20, n), device="cuda").t()
    for orig in (False, True):
        torch.testing.assert_close(H2.matvec(X, original_order=orig), H.matvec(X, original_order=orig), rtol=0,
                                   atol=0)
    # the loaded matrix stands on its own
    H.free()
    Y = H2.matvec(X)
    assert torch.isfinite(Y).all()


def test_load_refuses_other_cloud_and_damaged_files(hm, tmp_path):
    n = 12000
    pts, tree, st = cloud(hm, n, 6)
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_EXP, ell=0.1, tol=1e-5, max_rank=64)
    path = tmp_path / "h.bin"
    H.save(path)
    # same size, other points: the fingerprint differs
    pts2, tree2, st2 = cloud(hm, n, 7)
    with pytest.raises(hm.HMError) as e:
        hm.load_hmatrix(tree2, st2, path)
    assert e.value.status == 1
    # weak admissibility on the same tree: another structure
    stw = hm.construct_hmatrix_structure(tree, hm.WEAK, 1.0)
    with pytest.raises(hm.HMError):
        hm.load_hmatrix(tree, stw, path)
    data = path.read_bytes()
    short = tmp_path / "short.bin"
    short.write_bytes(data[: len(data) // 2])
    with pytest.raises(hm.HMError):
        hm.load_hmatrix(tree, st, short)
    junk = tmp_path / "junk.bin"
    junk.write_bytes(np.arange(1000, dtype=np.int32).tobytes())
    with pytest.raises(hm.HMError):
        hm.load_hmatrix(tree, st, junk)
    # the intact file still loads
    H2 = hm.load_hmatrix(tree, st, path)
    assert H2.stats()["num_lowrank"] == H.stats()["num_lowrank"]
