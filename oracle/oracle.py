"""ctypes wrapper of liboracle.so -- the CPU checker.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product (libhmb200.so and its Python
wrapper) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

K_EXP, K_MATERN32, K_GAUSS = 0, 1, 2

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "-s"], check=True)
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        i, dbl = ctypes.c_int, ctypes.c_double
        L.orc_tree_depth.argtypes = [i, i]
        L.orc_kdtree.argtypes = [i, i, i, P, P, P, P, P, P]
        L.orc_structure.argtypes = [i, i, i, dbl, P, P, P, P, P]
        L.orc_dense_rows_matvec.argtypes = [i, i, P, P, i, i, dbl, dbl, P, i, i, P, P]
        L.orc_dense_block.argtypes = [i, i, P, P, i, i, dbl, dbl, i, i, i, i, P]
        L.orc_block_error.argtypes = [i, i, P, P, i, i, dbl, dbl, i, i, i, i, i, P, P]
        L.orc_block_error.restype = dbl
        L.orc_kernel_r2.argtypes = [i, i, dbl, dbl]
        L.orc_kernel_r2.restype = dbl
        L.orc_dense_rows_block.argtypes = [i, i, P, P, i, i, dbl, dbl, P, i, i, i, P]
        L.orc_morton.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.orc_morton.restype = ctypes.c_uint32
        L.orc_blas_open.argtypes = [ctypes.c_char_p, i]
        L.orc_cpu_panel_matvec.argtypes = [i, i, P, P, i, dbl, dbl, i, i, i, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def tree_depth(n, bucket):
    return lib().orc_tree_depth(n, bucket)


def kdtree(points, n, d, bucket):
    """Restatement of constructKDTree (FULL_TREE).  points: SoA float64 [d*n].
    Returns dict(perm, offsets, bmin, bmax, split_dim, depth); boxes cover
    levels 0..depth, level l at [(2^l-1)*d]."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    depth = tree_depth(n, bucket)
    nleaf = 1 << depth
    perm = np.zeros(n, np.int32)
    offs = np.zeros(nleaf + 1, np.int32)
    bmin = np.zeros((2 * nleaf - 1) * d)
    bmax = np.zeros((2 * nleaf - 1) * d)
    sdim = np.zeros(max(nleaf - 1, 1), np.int32)
    rc = lib().orc_kdtree(n, d, bucket, _p(pts), _p(perm), _p(offs), _p(bmin), _p(bmax), _p(sdim))
    if rc:
        raise RuntimeError("orc_kdtree failed: %d" % rc)
    return dict(perm=perm, offsets=offs, bmin=bmin, bmax=bmax, split_dim=sdim[: nleaf - 1],
                depth=depth)


def structure(d, depth, admiss, eta, bmin, bmax, cap=None):
    """Restatement of constructHMatrixStructure.  Returns a list (levels
    1..depth) of int32 Morton arrays in the reference's order."""
    caps = []
    for lv in range(1, depth + 1):
        full = (1 << lv) * ((1 << lv) - 1)
        caps.append(full if cap is None else min(full, cap))
    bufs = [np.zeros(max(c, 1), np.int32) for c in caps]
    ptrs = (ctypes.c_void_p * max(depth, 1))(*[b.ctypes.data for b in bufs])
    counts = np.zeros(max(depth, 1), np.int32)
    capa = np.array(caps + [0], np.int32)
    rc = lib().orc_structure(d, depth, admiss, float(np.float32(eta)), _p(np.ascontiguousarray(bmin)),
                             _p(np.ascontiguousarray(bmax)), _p(counts), ptrs, _p(capa))
    if rc:
        raise RuntimeError("orc_structure failed: %d" % rc)
    return [bufs[lv][: counts[lv]].copy() for lv in range(depth)]


def morton(u, v):
    return lib().orc_morton(u, v)


def dense_rows_matvec(points, n, d, perm, kind, ell, nugget, rows, X, deriv=0):
    """FP64 Y[rows] = A[rows, :] X in tree order; X is (n, nrhs) column-major
    as a numpy array of shape (nrhs, n) or (n,)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    X = np.asarray(X, dtype=np.float64)
    nrhs = 1 if X.ndim == 1 else X.shape[0]
    Xc = np.ascontiguousarray(X.reshape(nrhs, n))
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    Y = np.zeros((nrhs, len(rows)))
    rc = lib().orc_dense_rows_matvec(n, d, _p(pts), _p(np.ascontiguousarray(perm, np.int32)), kind, deriv,
                                     ell, nugget, _p(rows), len(rows), nrhs, _p(Xc), _p(Y))
    if rc:
        raise RuntimeError("orc_dense_rows_matvec failed")
    return Y


def dense_block(points, n, d, perm, kind, ell, nugget, r0, m, c0, ncols, deriv=0):
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    out = np.zeros((ncols, m))
    lib().orc_dense_block(n, d, _p(pts), _p(np.ascontiguousarray(perm, np.int32)), kind, deriv, ell,
                          nugget, r0, m, c0, ncols, _p(out))
    return out.T  # (m, ncols)


def dense_rows_block(points, n, d, perm, kind, ell, nugget, rows, c0, ncols, deriv=0):
    """A[rows, c0:c0+ncols] in FP64 (rows: tree-order indices); shape (len(rows), ncols)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros((len(rows), ncols))
    lib().orc_dense_rows_block(n, d, _p(pts), _p(np.ascontiguousarray(perm, np.int32)), kind, deriv, ell, nugget,
                               _p(rows), len(rows), c0, ncols, _p(out))
    return out


def block_error(points, n, d, perm, kind, ell, nugget, r0, m, c0, ncols, U, V, deriv=0):
    """||A - U V^T||_F / ||A||_F for A = block (r0:r0+m, c0:c0+ncols)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    k = U.shape[1]
    Uc = np.asfortranarray(U, dtype=np.float64)
    Vc = np.asfortranarray(V, dtype=np.float64)
    return lib().orc_block_error(n, d, _p(pts), _p(np.ascontiguousarray(perm, np.int32)), kind, deriv,
                                 ell, nugget, r0, m, c0, ncols, k,
                                 Uc.ctypes.data_as(ctypes.c_void_p), Vc.ctypes.data_as(ctypes.c_void_p))


def kernel_r2(kind, r2, ell, deriv=0):
    return lib().orc_kernel_r2(kind, deriv, r2, ell)


def openblas_path():
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    for f in sorted(os.listdir(libdir)):
        if f.startswith("libscipy_openblas") and f.endswith(".so"):
            return os.path.join(libdir, f)
    raise FileNotFoundError("scipy's OpenBLAS not found")


def cpu_panel_matvec(points, n, d, perm, kind, ell, nugget, row0, nrows, X, threads, work=None):
    """Dense FP64 generation of rows [row0, row0+nrows) followed by OpenBLAS.
    Returns (Y (nrhs, nrows), t_gen, t_blas)."""
    L = lib()
    if L.orc_blas_open(openblas_path().encode(), threads):
        raise RuntimeError("cannot open OpenBLAS")
    X = np.asarray(X, dtype=np.float64)
    nrhs = 1 if X.ndim == 1 else X.shape[0]
    Xc = np.ascontiguousarray(X.reshape(nrhs, n))
    Y = np.zeros((nrhs, nrows))
    if work is None or work.size < nrows * n:
        work = np.empty(nrows * n)
    tg = ctypes.c_double()
    tb = ctypes.c_double()
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    rc = L.orc_cpu_panel_matvec(n, d, _p(pts), _p(np.ascontiguousarray(perm, np.int32)), kind, ell,
                                nugget, row0, nrows, nrhs, _p(Xc), _p(Y), _p(work), ctypes.byref(tg),
                                ctypes.byref(tb))
    if rc:
        raise RuntimeError("orc_cpu_panel_matvec failed")
    return Y, tg.value, tb.value
