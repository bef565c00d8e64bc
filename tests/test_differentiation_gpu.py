"""Differentiation form, checked through the C ABI.

L(x, l) = y^T H(l) x with H(l) the compressed Gaussian kernel matrix
exp(-r^2 / (2 l^2)).  dL/dx = H^T y is the adjoint product (hm_hmatvec with
trans = 1); dL/dl = y^T (dH/dl) x uses the derivative kernel dK/dl = K r^2/l^3
compressed on the same block structure, whose diagonal leaf blocks are
recomputed from the coordinates in every product instead of being stored.

torch.autograd.Function wraps the C ABI here only, as the gradient-check
harness: the library itself has no autograd dependency.  Checks: central
finite differences with step 1e-3 (in l, and along a direction in x), and an
FP64 dense gradient (oracle, src/expandMatrix.cu:142-231 restated with the
derivative kernel) on an 8192-point cloud.
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


class Problem:
    """One cloud, its tree and block structure; H(l) and dH/dl built on demand
    on that structure (cached per l)."""

    def __init__(self, hm, n, d=3, b=64, seed=17, tol=1e-5, max_rank=128):
        self.hm, self.n, self.d, self.tol, self.max_rank = hm, n, d, tol, max_rank
        self.pts = hm.generate_dataset(n, d, seed=seed)
        self.tree = hm.construct_kdtree(self.pts, n, d, b)
        self.st = hm.construct_hmatrix_structure(self.tree, hm.BOX_CENTER, 1.0)
        self.cache = {}

    def H(self, ell, deriv=0):
        key = (float(ell), deriv)
        if key not in self.cache:
            self.cache[key] = self.hm.build_hmatrix(self.tree, self.st, self.pts, kernel=self.hm.K_GAUSS,
                                                    ell=float(ell), tol=self.tol, max_rank=self.max_rank,
                                                    derivative=deriv, seed=3)
        return self.cache[key]


def make_hloss():
    import torch

    class HLoss(torch.autograd.Function):
        """L = sum(w * (H(l) x)) for fixed weights w: forward and backward both
        through hm_hmatvec."""

        @staticmethod
        def forward(ctx, x, ell, w, prob):
            H = prob.H(ell.item())
            hx = H.matvec(x)
            ctx.save_for_backward(x, ell, w)
            ctx.prob = prob
            return (w.double() * hx.double()).sum()

        @staticmethod
        def backward(ctx, gL):
            x, ell, w = ctx.saved_tensors
            prob = ctx.prob
            gx = prob.H(ell.item()).matvec(w, trans=1) * gL.float()        # adjoint product
            hdx = prob.H(ell.item(), deriv=1).matvec(x)                      # (dH/dl) x
            gl = (w.double() * hdx.double()).sum() * gL
            return gx, gl.reshape(ell.shape).to(device=ell.device, dtype=ell.dtype), None, None

    return HLoss


def test_gradients_match_central_differences(hm):
    """N = 2^17 uniform 3-D points, Gaussian l = 0.15, x and y ~ N(0,1)."""
    import torch

    n, ell0, h = 1 << 17, 0.15, 1e-3
    # The difference quotient divides the compression error of L by 2h: at
    # tol 1e-6 that is ~2e-5 of dL/dl, inside the 1e-4 bound below.
    prob = Problem(hm, n, tol=1e-6)
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn((n, 1), device="cuda", generator=gen).requires_grad_(True)
    w = torch.randn((n, 1), device="cuda", generator=gen)
    ell = torch.tensor([ell0], dtype=torch.float64, requires_grad=True)
    HLoss = make_hloss()
    L = HLoss.apply(x, ell, w, prob)
    L.backward()
    gl = ell.grad.item()
    # d/dl by central differences of the compressed loss (H rebuilt at l +- h)
    with torch.no_grad():
        Lp = HLoss.apply(x, torch.tensor([ell0 + h], dtype=torch.float64), w, prob).item()
        Lm = HLoss.apply(x, torch.tensor([ell0 - h], dtype=torch.float64), w, prob).item()
    fd = (Lp - Lm) / (2 * h)
    assert abs(gl - fd) <= 1e-4 * abs(fd), (gl, fd)
    # d/dx along a random direction v.  The adjoint first, exactly: the
    # bilinear identity v . (H^T w) = w . (H v) with one forward product.
    v = torch.randn((n, 1), device="cuda", generator=gen)
    gdx = (x.grad.double() * v.double()).sum().item()
    with torch.no_grad():
        whv = (w.double() * prob.H(ell0).matvec(v).double()).sum().item()
    assert abs(gdx - whv) <= 1e-5 * abs(whv), (gdx, whv)
    # Then central differences with step 1e-3.  L is linear in x, so dL/dx is
    # the same at every x; the quotient is taken at x0 = x / 100, where L is
    # 100 times smaller: at x itself |L| ~ 2e4 against a change of ~40 over
    # the step, and the products' FP32 rounding (~1e-6 of |L|, divided by
    # 2 step) alone would be ~2e-4 of the derivative.
    eps = 1e-3
    x0 = x.detach() / 100
    with torch.no_grad():
        Lp = HLoss.apply(x0 + eps * v, ell.detach(), w, prob).item()
        Lm = HLoss.apply(x0 - eps * v, ell.detach(), w, prob).item()
    fdx = (Lp - Lm) / (2 * eps)
    assert abs(gdx - fdx) <= 1e-4 * max(abs(fdx), 1e-12), (gdx, fdx)


def test_gradients_match_fp64_dense_on_8192_points(hm):
    import torch

    n, d, ell = 8192, 3, 0.15
    prob = Problem(hm, n, tol=1e-6, max_rank=64)
    perm = prob.tree.copy_out()["perm"]
    pts = prob.pts.cpu().numpy()
    rng = np.random.default_rng(8)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    xt = torch.from_numpy(x.astype(np.float32)).cuda().reshape(n, 1)
    yt = torch.from_numpy(y.astype(np.float32)).cuda().reshape(n, 1)
    rows = np.arange(n)
    # dL/dl = y^T (dK/dl) x, tree order on both sides
    ref_dx = oracle.dense_rows_matvec(pts, n, d, perm, oracle.K_GAUSS, ell, 0.0, rows, x[None, :], deriv=1)[0]
    gl_ref = float(y @ ref_dx)
    gl = float((yt.double() * prob.H(ell, deriv=1).matvec(xt).double()).sum())
    assert abs(gl - gl_ref) <= 1e-5 * np.abs(y) @ np.abs(ref_dx), (gl, gl_ref)
    # dL/dx = K^T y
    ref_ty = oracle.dense_rows_matvec(pts, n, d, perm, oracle.K_GAUSS, ell, 0.0, rows, y[None, :])[0]
    gx = prob.H(ell).matvec(yt, trans=1).cpu().numpy()[:, 0]
    assert np.linalg.norm(gx - ref_ty) <= 1e-5 * np.linalg.norm(ref_ty)


@pytest.mark.parametrize("precision", [0, 1])
def test_diagonal_from_coordinates_equals_stored(hm, precision):
    """The same matrix with its diagonal leaf blocks stored or recomputed from
    the coordinates in the product gives the same result (FP32 rounding)."""
    import torch

    n, d, b = 20000, 3, 64
    pts = hm.generate_dataset(n, d, seed=4)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0)
    kw = dict(kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=1e-4, max_rank=128, precision=precision, seed=9)
    Hs = hm.build_hmatrix(tree, st, pts, diag_from_coords=0, **kw)
    Hf = hm.build_hmatrix(tree, st, pts, diag_from_coords=1, **kw)
    assert Hf.stats()["num_dense"] < Hs.stats()["num_dense"]
    X = torch.randn((n, 7), device="cuda")
    Ys, Yf = Hs.matvec(X), Hf.matvec(X)
    rel = (torch.linalg.norm(Ys - Yf) / torch.linalg.norm(Ys)).item()
    # stored mixed diagonal blocks are BF16 hi + lo (about 2^-17 per entry)
    assert rel < (1e-6 if precision == 0 else 5e-6), rel
