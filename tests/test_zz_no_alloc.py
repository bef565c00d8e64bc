"""The allocation-free H-matvec (hm_hmatvec_noalloc), called through the C ABI.

It serves callers that may not allocate device memory when they apply the
operator (an external allocator owns all device memory, or a latency-bound
loop cannot afford a cudaMalloc that may synchronise the device).  Its scratch
is a fixed array in the library's device image; this file checks that two
calls in a row give the same product as hm_hmatvec, and that a matrix too
large for the fixed scratch is refused with a clear error.  The file name
makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hm():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hmatrix

    L = hmatrix.lib()
    L.hm_hmatvec_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return hmatrix


def _build(hm, n, d, b, tol, precision=0, seed=2024):
    pts = hm.generate_dataset(n, d, seed=seed)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    return hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=tol, max_rank=64,
                            precision=precision)


def _compare(hm, H, X, nrhs):
    """noalloc against hm_hmatvec on the same matrix and X; relative error."""
    import torch

    L = hm.lib()
    n = H.n
    Yref = torch.empty((nrhs, n), device="cuda", dtype=torch.float32)
    hm._check(L.hm_hmatvec(H.h, 0, nrhs, hm._ptr(X), n, hm._ptr(Yref), n, 0, None))
    Y = torch.full((nrhs, n), float("nan"), device="cuda", dtype=torch.float32)
    hm._check(L.hm_hmatvec_noalloc(H.h, nrhs, hm._ptr(X), n, hm._ptr(Y), n, None))
    torch.cuda.synchronize()
    return (torch.linalg.norm(Y - Yref) / torch.linalg.norm(Yref)).item()


def test_noalloc_matches_hmatvec_twice(hm):
    import torch

    n, nrhs = 4096, 16
    H = _build(hm, n, 3, 32, 1e-5)
    L = hm.lib()
    X = torch.randn((nrhs, n), device="cuda", dtype=torch.float32)  # column-major n x nrhs
    Yref = torch.empty_like(X)
    hm._check(L.hm_hmatvec(H.h, 0, nrhs, hm._ptr(X), n, hm._ptr(Yref), n, 0, None))
    for _ in range(2):  # the second call sees the first call's scratch contents
        Y = torch.full_like(X, float("nan"))
        hm._check(L.hm_hmatvec_noalloc(H.h, nrhs, hm._ptr(X), n, hm._ptr(Y), n, None))
        torch.cuda.synchronize()
        rel = (torch.linalg.norm(Y - Yref) / torch.linalg.norm(Yref)).item()
        assert rel < 1e-6, rel
    # a narrower call after a wider one
    Y3 = torch.empty((3, n), device="cuda", dtype=torch.float32)
    hm._check(L.hm_hmatvec_noalloc(H.h, 3, hm._ptr(X), n, hm._ptr(Y3), n, None))
    torch.cuda.synchronize()
    assert (torch.linalg.norm(Y3 - Yref[:3]) / torch.linalg.norm(Yref[:3])).item() < 1e-6


def test_noalloc_refuses_matrices_beyond_its_scratch(hm):
    import torch

    n = 1 << 16
    H = _build(hm, n, 3, 64, 1e-4)
    L = hm.lib()
    X = torch.randn((16, n), device="cuda", dtype=torch.float32)
    Y = torch.empty_like(X)
    st = L.hm_hmatvec_noalloc(H.h, 16, hm._ptr(X), n, hm._ptr(Y), n, None)
    assert st == 4  # HM_ERR_UNSUPPORTED
    msg = L.hm_last_error().decode()
    assert "static scratch holds" in msg and "16 MiB" in msg


def test_noalloc_mixed_form_after_another_layout(hm):
    """The mixed form's 16-column passes out of the static array.  A larger
    matrix with another layout runs first, so its projections, partials and X
    fragments are what the smaller matrix's calls find in the array: every word
    they read must be written by their own pass."""
    import torch

    big = _build(hm, 16384, 3, 64, 1e-4, precision=hm.PREC_MIXED, seed=77)
    small = _build(hm, 4096, 3, 32, 1e-4, precision=hm.PREC_MIXED)
    Xb = torch.randn((20, big.n), device="cuda", dtype=torch.float32)
    assert _compare(hm, big, Xb, 20) < 1e-6
    Xs = torch.randn((16, small.n), device="cuda", dtype=torch.float32)
    for nrhs in (16, 16, 3):
        assert _compare(hm, small, Xs, nrhs) < 1e-6


def test_noalloc_refuses_a_mixed_matrix_beyond_its_scratch(hm):
    """The mixed form needs 16 floats per point for its X fragments, so 2^18
    points are beyond the 16 MiB array whatever the ranks."""
    import torch

    n = 1 << 18
    H = _build(hm, n, 3, 64, 1e-4, precision=hm.PREC_MIXED)
    L = hm.lib()
    X = torch.randn((16, n), device="cuda", dtype=torch.float32)
    Y = torch.empty_like(X)
    assert L.hm_hmatvec_noalloc(H.h, 16, hm._ptr(X), n, hm._ptr(Y), n, None) == 4
    msg = L.hm_last_error().decode()
    assert "mixed form" in msg and "16 per point" in msg and "16 MiB" in msg
