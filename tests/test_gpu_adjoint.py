"""Adjoint of the FMM through torch.autograd on the full C4 shape:
1,048,576 + 1,048,576 uniform points in the unit cube, weights N(0,1),
Gaussian exp(-r^2/0.01), 5 nodes per dimension, Depth 6 (leaves of ~32
points), loss L = sum_i g_i c_i with g N(0,1).

The adjoint is the exact derivative of the FMM's own result: the transposed
FMM for dL/dw (the FMM is linear in w), the differentiated L2P interpolant of
the transposed field (= P2M^T) plus grad f for dL/dy, the differentiated L2P
of the forward field plus grad f for dL/dx.  Checks:

* finite differences of the FMM result on 64 random coordinates per input:
  central differences at eps = 1e-3 and 5e-4 combined by Richardson
  extrapolation, (4 D(eps/2) - D(eps)) / 3, which cancels the (eps/sigma)^2
  term of the central difference (~2e-5 here) and leaves O((eps/sigma)^4)
  ~ 1e-8.  A coordinate whose +-eps perturbation would move its point to
  another leaf (the FMM is piecewise smooth across leaf faces) is redrawn;
  at most 12 redraws per input are allowed (~4 expected).
  Bar: max |adjoint - FD| <= 1e-5 of the largest |FD| for dL/dw, dL/dx and
  dL/dy.  The raw eps = 1e-3 central difference is checked too, at the
  tolerance its truncation error allows (1e-4).
* the exact solver's analytic gradient: within 10x the FMM's own relative
  error on the potential (5 nodes interpolate this Gaussian to ~2e-4), for
  the plain FP64 path and both mixed precisions (TF32x3, BF16x3);
* finite differences of the exact sum against the exact gradient
  (validates the grad f kernels), <= 1e-5 of the largest (Richardson).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

N = 1 << 20
EPS = 1e-3
DEPTH = 6
PO = 4
PROBES = 64
MAX_REDRAWS = 12


@pytest.fixture(scope="module")
def problem():
    import torch
    r = np.random.default_rng(4)
    x = torch.tensor(r.random((N, 3)), dtype=torch.float64, device="cuda", requires_grad=True)
    y = torch.tensor(r.random((N, 3)), dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.tensor(r.standard_normal(N), dtype=torch.float64, device="cuda", requires_grad=True)
    g = torch.tensor(r.standard_normal(N), dtype=torch.float64, device="cuda")
    return x, y, w, g


def _grads(problem, precision="fp64"):
    import pyfmma
    from pyfmma.torch import fmm
    x, y, w, g = problem
    for t in (x, y, w):
        t.grad = None
    c = fmm(x, y, w, kernel=pyfmma.kernels.gaussian(0.01), poly_ord=PO, depth=DEPTH, precision=precision)
    (g * c).sum().backward()
    return c.detach(), x.grad.detach().clone(), y.grad.detach().clone(), w.grad.detach().clone()


class _Fd:
    """Central differences of L = g . c through the FMM on device tensors;
    each difference is g . (c+ - c-), so entries that do not move cancel
    exactly."""

    def __init__(self, ctx, X, Y, W, G):
        self.ctx, self.X, self.Y, self.W, self.G = ctx, X, Y, W, G

    def _c(self, X, Y, W):
        c, _ = self.ctx.solve(X, Y, W, poly_ord=PO, depth=DEPTH)
        return c

    def central(self, which, i, q, h):
        import torch
        args = {"x": self.X, "y": self.Y, "w": self.W}
        base = args[which]
        plus, minus = base.clone(), base.clone()
        if which == "w":
            plus[i] += h
            minus[i] -= h
        else:
            plus[i, q] += h
            minus[i, q] -= h
        cp = self._c(*(plus if k == which else args[k] for k in "xyw"))
        cm = self._c(*(minus if k == which else args[k] for k in "xyw"))
        return float(torch.dot(self.G, cp - cm)) / (2 * h)

    def richardson(self, which, i, q):
        d1 = self.central(which, i, q, EPS)
        d2 = self.central(which, i, q, EPS / 2)
        return (4 * d2 - d1) / 3, d1


def _leaf_safe(P, i, q, origin, length, h):
    """True when P[i, q] +- h stays in its leaf and inside the cube's extent
    (the cube, and so every leaf, is unchanged)."""
    nb = 1 << (DEPTH - 1)
    wdt = length / nb
    u = (P[i, q] - origin[q]) / wdt
    k = np.floor(u)
    return (u - h / wdt > k) and (u + h / wdt < k + 1) and (P[i, q] - h > origin[q]) and \
        (P[i, q] + h < origin[q] + length)


def test_adjoint_matches_fd_of_the_fmm(ctx, problem):
    _, dx, dy, dw = _grads(problem)
    dx, dy, dw = dx.cpu().numpy(), dy.cpu().numpy(), dw.cpu().numpy()
    x, y, w, g = problem
    X, Y, W, G = (t.detach().clone() for t in (x, y, w, g))
    Xh, Yh = X.cpu().numpy(), Y.cpu().numpy()
    ctx.set_kernel("gaussian", 0.01)
    _, _, origin, length = ctx.tree_export(Xh, Yh, DEPTH)
    # the cube's extremes are never probed (a moved extreme would move the cube)
    fd = _Fd(ctx, X, Y, W, G)
    r = np.random.default_rng(9)
    res = {"dx": [], "dy": [], "dw": []}
    redraws = {"dx": 0, "dy": 0}
    for i in r.choice(N, PROBES, replace=False):
        ext, raw = fd.richardson("w", int(i), 0)
        res["dw"].append((dw[i], ext, raw))
    for name, P, grad, which in (("dx", Xh, dx, "x"), ("dy", Yh, dy, "y")):
        while len(res[name]) < PROBES:
            i, q = int(r.integers(0, N)), int(r.integers(0, 3))
            if not _leaf_safe(P, i, q, origin, length, EPS):
                redraws[name] += 1
                continue
            ext, raw = fd.richardson(which, i, q)
            res[name].append((grad[i, q], ext, raw))
    assert redraws["dx"] <= MAX_REDRAWS and redraws["dy"] <= MAX_REDRAWS, redraws
    for name in ("dw", "dx", "dy"):
        a = np.array(res[name])
        scale = np.max(np.abs(a[:, 1]))
        err_ext = np.max(np.abs(a[:, 0] - a[:, 1])) / scale
        err_raw = np.max(np.abs(a[:, 0] - a[:, 2])) / scale
        print(f"{name}: max|adj - FD| / max|FD| = {err_ext:.2e} (Richardson), {err_raw:.2e} (eps = 1e-3)")
        assert err_ext <= 1e-5, (name, err_ext, err_raw)
        assert err_raw <= 1e-4, (name, err_raw)


@pytest.mark.parametrize("precision", ["fp64", "tf32x3", "bf16x3"])
def test_adjoint_close_to_exact_gradient(ctx, problem, precision):
    import torch
    c, dx, dy, dw = _grads(problem, precision)
    x, y, w, g = problem
    X, Y, W, G = (t.detach() for t in (x, y, w, g))
    ctx.set_kernel("gaussian", 0.01)
    # the exact sums on 4096 sampled targets / sources (all 2^20 would be 10^12 pairs)
    rows = np.sort(np.random.default_rng(12).choice(N, 4096, replace=False))
    ri = torch.from_numpy(rows).cuda()
    ce, cg, _ = ctx.solve_grad(X[ri].contiguous(), Y, W, solver="exact")
    u, ug, _ = ctx.solve_grad(Y[ri].contiguous(), X, G, solver="exact")
    e_pot = rel_l2(c[ri].cpu().numpy(), ce.cpu().numpy())
    assert e_pot <= 1e-3
    for got, want, name in ((dx[ri], G[ri].unsqueeze(-1) * cg, "dx"), (dy[ri], W[ri].unsqueeze(-1) * ug, "dy"),
                            (dw[ri], u, "dw")):
        e = rel_l2(got.cpu().numpy(), want.cpu().numpy())
        assert e <= 10 * e_pot, (precision, name, e, e_pot)


def test_exact_gradient_matches_fd_of_exact_sum(ctx):
    r = np.random.default_rng(10)
    n = 65536
    X, Y, W = r.random((n, 3)), r.random((n, 3)), r.standard_normal(n)
    ctx.set_kernel("gaussian", 0.01)
    rows = r.choice(n, 64, replace=False)
    _, cg, _ = ctx.solve_grad(X, Y, W, solver="exact")

    def d(i, q, h):
        xp, xm = X.copy(), X.copy()
        xp[i, q] += h
        xm[i, q] -= h
        return (ctx.exact_rows([i], xp, Y, W)[0] - ctx.exact_rows([i], xm, Y, W)[0]) / (2 * h)

    pairs = []
    for i, q in zip(rows, r.integers(0, 3, 64)):
        pairs.append((cg[i, q], (4 * d(i, q, EPS / 2) - d(i, q, EPS)) / 3))
    a = np.array(pairs)
    assert np.max(np.abs(a[:, 0] - a[:, 1])) / np.max(np.abs(a[:, 1])) <= 1e-5
