"""Python host binding of libhmb200.so (ctypes over the C ABI in include/hm.h).

Mirrors the reference's pipeline operators (reference file:line):

    generate_dataset            generateDataset            src/generateDataset.cu:15-19
    construct_kdtree            allocateKDTree +           src/kDTree.cu:6-31,
                                constructKDTree            src/kDTreeConstruction.cu:14-231
    construct_hmatrix_structure constructHMatrixStructure  src/HMatrixStructure.cu:133-160
    build_hmatrix               allocateHMatrix +          src/HMatrix.cu:57-103,
                                generateHMatrixFromStruct  src/constructHMatrixFromStruct.cu:13-103
    HMatrix.matvec              HMatrixVecMult             src/HMatrixVectorMultiplication.cu:10-27

Device memory comes from torch tensors (plumbing only); all computation runs in
the CUDA kernels of libhmb200.so.  There is no fallback: if the library is
missing the import-time loader raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhmb200.so")

WEAK, BOX_CENTER = 0, 1
K_EXP, K_MATERN32, K_GAUSS = 0, 1, 2
PREC_FP32, PREC_MIXED = 0, 1


class HMError(RuntimeError):
    """A libhmb200 call returned a non-zero hm_status."""

    def __init__(self, status, msg):
        super().__init__("hm status %d: %s" % (status, msg))
        self.status = status


class BuildOpts(ctypes.Structure):
    _fields_ = [
        ("kernel", ctypes.c_int),
        ("ell", ctypes.c_double),
        ("nugget", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("max_rank", ctypes.c_int),
        ("leaf_max_rank", ctypes.c_int),
        ("sample_block", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("derivative", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("diag_from_coords", ctypes.c_int),
        ("level_schedule", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("num_lowrank", ctypes.c_longlong),
        ("num_dense", ctypes.c_longlong),
        ("rank_sum", ctypes.c_longlong),
        ("max_rank_seen", ctypes.c_int),
        ("factor_bytes", ctypes.c_longlong),
        ("dense_bytes", ctypes.c_longlong),
        ("num_unconverged", ctypes.c_longlong),
        ("mixed_bytes", ctypes.c_longlong),
        ("build_seconds", ctypes.c_double),
        ("num_split", ctypes.c_longlong),
        ("device_bytes", ctypes.c_longlong),
        ("phase_seconds", ctypes.c_double * 8),
    ]

    PHASES = ("setup", "sketch", "orth", "projection", "truncation", "diagonal", "panels", "plan")


_lib = None


def lib():
    """Load libhmb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libhmb200.so not built: run `make -C %s`" % HERE)
        L = ctypes.CDLL(LIB_PATH)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.hm_last_error.restype = ctypes.c_char_p
        L.hm_version.restype = ctypes.c_char_p
        L.hm_generate_dataset.argtypes = [I, I, ctypes.c_ulonglong, P, P]
        L.hm_generate_mixture.argtypes = [I, I, I, D, D, ctypes.c_ulonglong, P, P]
        L.hm_kdtree_build.argtypes = [P, I, I, I, P, ctypes.POINTER(P)]
        L.hm_kdtree_info.argtypes = [P, P, P, P, P]
        L.hm_kdtree_copy_out.argtypes = [P, P, P, P, P, P]
        L.hm_kdtree_device_perm.argtypes = [P]
        L.hm_kdtree_device_perm.restype = P
        L.hm_kdtree_free.argtypes = [P]
        L.hm_structure_build.argtypes = [P, I, D, P, ctypes.POINTER(P)]
        L.hm_structure_info.argtypes = [P, P, P]
        L.hm_structure_tiles.argtypes = [P, I, P]
        L.hm_structure_jds.argtypes = [P, I, P, P, P, P, P, P]
        L.hm_structure_free.argtypes = [P]
        if hasattr(L, "hm_hmatrix_build"):
            L.hm_build_opts_default.argtypes = [I, ctypes.POINTER(BuildOpts)]
            L.hm_hmatrix_build.argtypes = [P, P, P, ctypes.POINTER(BuildOpts), P, ctypes.POINTER(P)]
            L.hm_hmatrix_build_rows.argtypes = [P, P, P, ctypes.POINTER(BuildOpts), I, I, P, ctypes.POINTER(P)]
            L.hm_hmatvec_f64.argtypes = [P, I, I, P, I, P, I, I, P]
            L.hm_kdtree_build_div.argtypes = [P, I, I, I, I, P, ctypes.POINTER(P)]
            L.hm_hmatrix_stats_get.argtypes = [P, ctypes.POINTER(Stats)]
            L.hm_hmatrix_check.argtypes = [P, P]
            L.hm_hmatvec.argtypes = [P, I, I, P, I, P, I, I, P]
            L.hm_hmatrix_free.argtypes = [P]
            L.hm_hmatrix_blocks.argtypes = [P, P, P, P, P]
            L.hm_hmatrix_block_factors.argtypes = [P, I, P, P]
            L.hm_hmatvec_kernels.argtypes = [P, I, P, I, P, I, P, I, P, P, P, P]
            L.hm_batch_create.argtypes = [I, P, P, P, ctypes.POINTER(P)]
            L.hm_batch_info.argtypes = [P, P, P, P, P]
            L.hm_batch_build.argtypes = [P, ctypes.POINTER(BuildOpts), P]
            L.hm_batch_hmatrix.argtypes = [P]
            L.hm_batch_hmatrix.restype = P
            L.hm_batch_matvec.argtypes = [P, I, P, I, P, I, I, P]
            L.hm_batch_free.argtypes = [P]
            L.hm_autotune.argtypes = [P, I, ctypes.c_char_p, P, P, ctypes.c_char_p, I]
            L.hm_schedule_set.argtypes = [P, ctypes.c_char_p, P]
            L.hm_cg_solve.argtypes = [P, I, P, I, P, I, D, I, I, P, P, P]
            L.hm_hmatrix_save.argtypes = [P, ctypes.c_char_p]
            L.hm_hmatrix_load.argtypes = [P, P, ctypes.c_char_p, P, ctypes.POINTER(P)]
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise HMError(status, lib().hm_last_error().decode())


def _check_vectors(X, n, name):
    """The C ABI takes raw pointers and trusts the sizes it is given: a block
    of vectors must be a float32 CUDA tensor of shape (n, nrhs)."""
    if X.dim() != 2 or X.shape[0] != n or X.shape[1] < 1:
        raise ValueError("%s must have shape (%d, nrhs), got %s" % (name, n, tuple(X.shape)))
    if str(X.dtype) != "torch.float32" or X.device.type != "cuda":
        raise ValueError("%s must be a float32 CUDA tensor" % name)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def version():
    return lib().hm_version().decode()


def generate_dataset(n, d, seed=1234, out=None, stream=None):
    """Points in SoA layout p[dim*n + i] (float64 CUDA tensor of n*d)."""
    import torch

    if out is None:
        out = torch.empty(n * d, dtype=torch.float64, device="cuda")
    _check(lib().hm_generate_dataset(n, d, seed, _ptr(out), _stream(stream)))
    return out


class KDTree:
    """Handle of a device KD tree (FULL_TREE division)."""

    def __init__(self, handle):
        self.h = handle
        n, d, b, depth = (ctypes.c_int() for _ in range(4))
        _check(lib().hm_kdtree_info(self.h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(b),
                                    ctypes.byref(depth)))
        self.n, self.d, self.bucket, self.depth = n.value, d.value, b.value, depth.value

    def copy_out(self):
        """Host copies: perm, offsets, bmin, bmax (levels 0..depth), split_dim."""
        nleaf = 1 << self.depth
        perm = np.zeros(self.n, np.int32)
        offs = np.zeros(nleaf + 1, np.int32)
        bmin = np.zeros((2 * nleaf - 1) * self.d)
        bmax = np.zeros((2 * nleaf - 1) * self.d)
        sdim = np.zeros(max(nleaf - 1, 1), np.int32)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        _check(lib().hm_kdtree_copy_out(self.h, P(perm), P(offs), P(bmin), P(bmax), P(sdim)))
        return dict(perm=perm, offsets=offs, bmin=bmin, bmax=bmax, split_dim=sdim[: nleaf - 1])

    def free(self):
        if self.h:
            lib().hm_kdtree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=1, out=None, stream=None):
    """Points of an isotropic Gaussian mixture (hm_generate_mixture), SoA float64."""
    import torch

    if out is None:
        out = torch.empty(n * d, dtype=torch.float64, device="cuda")
    _check(lib().hm_generate_mixture(n, d, ncomp, sigma_min, sigma_max, seed, _ptr(out), _stream(stream)))
    return out


def construct_kdtree(points, n, d, bucket, stream=None):
    h = ctypes.c_void_p()
    _check(lib().hm_kdtree_build(_ptr(points), n, d, bucket, _stream(stream), ctypes.byref(h)))
    return KDTree(h)


class Structure:
    def __init__(self, handle, tree):
        self.h = handle
        self.tree = tree  # keeps the tree alive
        nl = ctypes.c_int()
        _check(lib().hm_structure_info(self.h, ctypes.byref(nl), None))
        self.num_levels = nl.value
        self.depth = self.num_levels - 1
        counts = np.zeros(max(self.depth, 1), np.int32)
        _check(lib().hm_structure_info(self.h, None, counts.ctypes.data_as(ctypes.c_void_p)))
        self.counts = counts[: self.depth]

    def tiles(self, level):
        out = np.zeros(max(int(self.counts[level - 1]), 1), np.int32)
        _check(lib().hm_structure_tiles(self.h, level, out.ctypes.data_as(ctypes.c_void_p)))
        return out[: self.counts[level - 1]]

    def all_tiles(self):
        return [self.tiles(lv) for lv in range(1, self.depth + 1)]

    def jds(self, level):
        nrows = 1 << level
        nb = int(self.counts[level - 1])
        maxc = ctypes.c_int()
        _check(lib().hm_structure_jds(self.h, level, None, None, None, None, None, ctypes.byref(maxc)))
        rp = np.zeros(nrows + 1, np.int32)
        cb = np.zeros(max(nb, 1), np.int32)
        jr = np.zeros(nrows, np.int32)
        jp = np.zeros(maxc.value + 1, np.int32)
        jb = np.zeros(max(nb, 1), np.int32)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        _check(lib().hm_structure_jds(self.h, level, P(rp), P(cb), P(jr), P(jp), P(jb), None))
        return dict(row_ptr=rp, csr_blk=cb[:nb], jds_rows=jr, jds_ptr=jp, jds_blk=jb[:nb],
                    max_row_blocks=maxc.value)

    def free(self):
        if self.h:
            lib().hm_structure_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def construct_hmatrix_structure(tree, admissibility=BOX_CENTER, eta=1.0, stream=None):
    h = ctypes.c_void_p()
    _check(lib().hm_structure_build(tree.h, admissibility, eta, _stream(stream), ctypes.byref(h)))
    return Structure(h, tree)


class HMatrix:
    """Handle of a built H-matrix (keeps its tree and structure alive)."""

    def __init__(self, handle, tree, structure):
        self.h = handle
        self.tree = tree
        self.structure = structure
        self.n = tree.n

    def save(self, path):
        """Write the H-matrix to a binary file (hm_hmatrix_save)."""
        _check(lib().hm_hmatrix_save(self.h, str(path).encode()))

    def stats(self):
        st = Stats()
        _check(lib().hm_hmatrix_stats_get(self.h, ctypes.byref(st)))
        out = {k: getattr(st, k) for k, _ in Stats._fields_ if k != "phase_seconds"}
        out["phase_seconds"] = dict(zip(Stats.PHASES, list(st.phase_seconds)))
        return out

    def check(self, stream=None):
        """Wait for the stream and raise if a bounded device-side wait of a
        product kernel gave up since the last check (hm_hmatrix_check)."""
        _check(lib().hm_hmatrix_check(self.h, _stream(stream)))

    def matvec(self, X, Y=None, trans=0, original_order=False, stream=None):
        """Y = H X for a float32 CUDA tensor X of shape (n, nrhs), column-major
        (i.e. X.T contiguous) or a contiguous (n,) vector."""
        import torch

        n = self.n
        if X.dim() == 1:
            X = X[:, None]
        _check_vectors(X, n, "X")
        nrhs = X.shape[1]
        Xc = X.t().contiguous() if not X.t().is_contiguous() else X.t()
        if Y is None:
            Yc = torch.empty((nrhs, n), dtype=torch.float32, device=X.device)
        else:
            _check_vectors(Y, n, "Y")
            if Y.shape[1] != nrhs:
                raise ValueError("Y must have as many columns as X")
            Yc = Y.t()
            assert Yc.is_contiguous()
        _check(lib().hm_hmatvec(self.h, trans, nrhs, _ptr(Xc), n, _ptr(Yc), n, 1 if original_order else 0,
                                _stream(stream)))
        return Yc.t()

    def matvec_f64(self, X, Y=None, trans=0, original_order=False, stream=None):
        """hm_hmatvec_f64: the reference's FP64 vectors, X a float64 CUDA
        tensor (n, nrhs) with X.T contiguous; narrowed and widened on the
        device."""
        import torch

        n = self.n
        if X.dim() == 1:
            X = X[:, None]
        if X.dim() != 2 or X.shape[0] != n or X.dtype != torch.float64 or X.device.type != "cuda":
            raise ValueError("X must be a float64 CUDA tensor of shape (%d, nrhs)" % n)
        nrhs = X.shape[1]
        Xc = X.t().contiguous()
        Yc = torch.empty((nrhs, n), dtype=torch.float64, device=X.device) if Y is None else Y.t()
        assert Yc.is_contiguous() and Yc.shape == (nrhs, n)
        _check(lib().hm_hmatvec_f64(self.h, trans, nrhs, _ptr(Xc), n, _ptr(Yc), n, 1 if original_order else 0,
                                    _stream(stream)))
        return Yc.t()

    def blocks(self):
        """Host copy of the block list: (lowrank rows [r0, m, c0, n, k, level],
        dense rows [r0, m, c0, n, transposed]), both orientations."""
        nl, nd = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().hm_hmatrix_blocks(self.h, ctypes.byref(nl), ctypes.byref(nd), None, None))
        lr = np.zeros((max(nl.value, 1), 6), np.int32)
        de = np.zeros((max(nd.value, 1), 5), np.int32)
        _check(lib().hm_hmatrix_blocks(self.h, None, None, lr.ctypes.data_as(ctypes.c_void_p),
                                       de.ctypes.data_as(ctypes.c_void_p)))
        return lr[: nl.value], de[: nd.value]

    def block_factors(self, i):
        """U (m x k) and V (n x k) of low-rank block i, float64 numpy."""
        lr, _ = self.blocks()
        r0, m, c0, n, k, lvl = lr[i]
        U = np.zeros(m * max(k, 1), np.float32)
        V = np.zeros(n * max(k, 1), np.float32)
        _check(lib().hm_hmatrix_block_factors(self.h, i, U.ctypes.data_as(ctypes.c_void_p),
                                              V.ctypes.data_as(ctypes.c_void_p)))
        return (U[: m * k].reshape(k, m).T.astype(np.float64), V[: n * k].reshape(k, n).T.astype(np.float64))

    def free(self):
        if self.h and getattr(self, "owned", True):
            lib().hm_hmatrix_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """Independent clouds joined as one forest (hm_batch_*): one build for all
    clouds, one graph-launched product over the concatenated rows."""

    def __init__(self, trees, structures, stream=None):
        n = len(trees)
        self.trees, self.structures = list(trees), list(structures)  # kept alive
        val = lambda h: h.value if isinstance(h, ctypes.c_void_p) else h
        th = (ctypes.c_void_p * n)(*[val(t.h) for t in trees])
        sh = (ctypes.c_void_p * n)(*[val(s.h) for s in structures])
        h = ctypes.c_void_p()
        _check(lib().hm_batch_create(n, th, sh, _stream(stream), ctypes.byref(h)))
        self.h = h
        nc, nt, dep = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        offs = (ctypes.c_int * (n + 1))()
        _check(lib().hm_batch_info(self.h, ctypes.byref(nc), ctypes.byref(nt), ctypes.byref(dep), offs))
        self.nclouds, self.n, self.depth = nc.value, nt.value, dep.value
        self.row_offsets = list(offs)

    def build(self, kernel=K_EXP, ell=None, nugget=0.0, tol=1e-5, max_rank=64, leaf_max_rank=0, sample_block=16,
              precision=PREC_FP32, derivative=0, seed=0, stream=None, diag_from_coords=-1):
        o = default_opts(self.trees[0].d)
        o.kernel, o.nugget, o.tol, o.max_rank = kernel, nugget, tol, max_rank
        if ell is not None:
            o.ell = ell
        o.leaf_max_rank, o.sample_block, o.precision = leaf_max_rank, sample_block, precision
        o.derivative, o.seed, o.diag_from_coords = derivative, seed, diag_from_coords
        _check(lib().hm_batch_build(self.h, ctypes.byref(o), _stream(stream)))

    def hmatrix(self):
        """The batch's H-matrix (owned by the batch)."""
        H = HMatrix(lib().hm_batch_hmatrix(self.h), self, None)
        H.owned = False
        return H

    def matvec(self, X, Y, stream, original_order=False):
        """Y = H X over all clouds through the recorded CUDA graph; X, Y float32
        CUDA tensors (n_total, nrhs) with X.T, Y.T contiguous; stream: a
        torch.cuda.Stream (not the legacy default stream)."""
        Xc, Yc = X.t(), Y.t()
        assert Xc.is_contiguous() and Yc.is_contiguous()
        _check(lib().hm_batch_matvec(self.h, X.shape[1], _ptr(Xc), self.n, _ptr(Yc), self.n,
                                     1 if original_order else 0, _stream(stream)))
        return Y

    def free(self):
        if self.h:
            lib().hm_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def autotune(H, nrhs=16, cache_path=None, stream=None):
    """Pick the fastest product schedule for H (hm_autotune); returns
    (description, taken_from_cache)."""
    fc = ctypes.c_int()
    buf = ctypes.create_string_buffer(128)
    _check(lib().hm_autotune(H.h, nrhs, cache_path.encode() if cache_path else None, _stream(stream),
                             ctypes.byref(fc), buf, 128))
    return buf.value.decode(), bool(fc.value)


def cg_solve(H, B, tol=1e-6, max_iter=1000, check_every=8, stream=None):
    """Solve H X = B by conjugate gradients (hm_cg_solve), tree order.  B: a
    float32 CUDA tensor (n, nrhs) with B.T contiguous, or (n,).  Returns (X,
    iterations, worst true relative residual); raises HMError with status 6
    when max_iter iterations do not reach tol."""
    import torch

    n = H.n
    if B.dim() == 1:
        B = B[:, None]
    _check_vectors(B, n, "B")
    nrhs = B.shape[1]
    Bc = B.t().contiguous() if not B.t().is_contiguous() else B.t()
    Xc = torch.empty((nrhs, n), dtype=torch.float32, device=B.device)
    it, res = ctypes.c_int(), ctypes.c_double()
    _check(lib().hm_cg_solve(H.h, nrhs, _ptr(Bc), n, _ptr(Xc), n, tol, max_iter, check_every, _stream(stream),
                             ctypes.byref(it), ctypes.byref(res)))
    return Xc.t(), it.value, res.value


class PiecewiseHMatrix:
    """An H-matrix kept out of device memory, in block-row pieces.

    The rows are split into `pieces` runs of whole subtrees
    (ranks.subtree_shards).  Each piece -- the blocks whose rows or columns
    touch its rows (hm_hmatrix_build_rows) -- is built on the device, written
    to a file in `directory` and freed, so the device never holds more than
    one piece.  matvec() loads the pieces one at a time, multiplies all of X
    and keeps each piece's rows.  A product costs `pieces` file reads and
    panel rebuilds on top of the arithmetic: a way past the device's memory,
    not a fast path.  (The reference's large-matrix variant treats its matrix
    in p x p pieces; here a piece is a whole block row, whose blocks a product
    needs together.)"""

    def __init__(self, tree, structure, points, pieces, directory, stream=None, **build_kw):
        import ranks

        self.tree, self.structure, self.n = tree, structure, tree.n
        self.shards = ranks.subtree_shards(tree.copy_out()["offsets"], pieces)
        self.paths, self.piece_device_bytes = [], []
        for i, (lb, le, r0, r1) in enumerate(self.shards):
            H = build_hmatrix(tree, structure, points, leaves=(lb, le), stream=stream, **build_kw)
            self.piece_device_bytes.append(H.stats()["device_bytes"])
            path = os.path.join(str(directory), "piece_%d_of_%d.hmb" % (i, pieces))
            H.save(path)
            H.free()
            self.paths.append(path)

    def matvec(self, X, stream=None):
        """Y = H X for a float32 CUDA tensor X (n, nrhs) (X.T contiguous), tree order."""
        import torch

        _check_vectors(X, self.n, "X")
        nrhs = X.shape[1]
        Y = torch.empty((nrhs, self.n), dtype=torch.float32, device=X.device).t()
        Yp = torch.empty((nrhs, self.n), dtype=torch.float32, device=X.device).t()
        for (lb, le, r0, r1), path in zip(self.shards, self.paths):
            H = load_hmatrix(self.tree, self.structure, path, stream=stream)
            H.matvec(X, Y=Yp, stream=stream)
            Y[r0:r1] = Yp[r0:r1]
            H.free()
        return Y


def load_hmatrix(tree, structure, path, stream=None):
    """Read an H-matrix written by HMatrix.save (hm_hmatrix_load); tree and
    structure must be the ones it was built on."""
    h = ctypes.c_void_p()
    _check(lib().hm_hmatrix_load(tree.h, structure.h, str(path).encode(), _stream(stream), ctypes.byref(h)))
    return HMatrix(h, tree, structure)


def schedule_set(H, choice, stream=None):
    """Apply a schedule in hm_autotune's notation (hm_schedule_set)."""
    _check(lib().hm_schedule_set(H.h, choice.encode(), _stream(stream)))


def default_opts(d):
    o = BuildOpts()
    lib().hm_build_opts_default(d, ctypes.byref(o))
    return o


def build_hmatrix(tree, structure, points=None, kernel=K_EXP, ell=None, nugget=0.0, tol=1e-5, max_rank=64,
                  leaf_max_rank=0, sample_block=16, precision=PREC_FP32, derivative=0, seed=0, stream=None,
                  diag_from_coords=-1, leaves=None, level_schedule=0):
    """hm_hmatrix_build; with leaves=(leaf_begin, leaf_end), the block-row
    shard of those leaves' rows (hm_hmatrix_build_rows)."""
    o = default_opts(tree.d)
    o.kernel = kernel
    if ell is not None:
        o.ell = ell
    o.nugget = nugget
    o.tol = tol
    o.max_rank = max_rank
    o.leaf_max_rank = leaf_max_rank
    o.sample_block = sample_block
    o.precision = precision
    o.derivative = derivative
    o.seed = seed
    o.diag_from_coords = diag_from_coords
    o.level_schedule = level_schedule
    h = ctypes.c_void_p()
    pp = _ptr(points) if points is not None else None
    if leaves is None:
        _check(lib().hm_hmatrix_build(tree.h, structure.h, pp, ctypes.byref(o), _stream(stream), ctypes.byref(h)))
    else:
        _check(lib().hm_hmatrix_build_rows(tree.h, structure.h, pp, ctypes.byref(o), int(leaves[0]),
                                           int(leaves[1]), _stream(stream), ctypes.byref(h)))
    return HMatrix(h, tree, structure)


# reference-style aliases
generateDataset = generate_dataset
constructKDTree = construct_kdtree
constructHMatrixStructure = construct_hmatrix_structure
generateHMatrixFromStruct = build_hmatrix
