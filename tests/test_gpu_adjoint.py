"""Adjoint of the FMM through torch.autograd on the C4 shape reduced to
65,536 + 65,536 uniform points in the unit cube, Gaussian exp(-r^2/0.01),
5 nodes per dimension, Depth 6 (leaf width 1/32, as in C4).

The adjoint is the exact derivative of the FMM's own result: the transposed
FMM for dL/dw (the FMM is linear in w), the differentiated L2P interpolant of
the transposed field (= P2M^T) plus grad f for dL/dy, the differentiated L2P
of the forward field plus grad f for dL/dx.  Checks:

* central finite differences of the FMM result (eps = 1e-3, 64 random
  coordinates per input; coordinates whose perturbation moves a point to
  another leaf are skipped, the FMM being piecewise smooth there):
  max |adjoint - FD| <= 1e-5 of the largest |FD| for dL/dw, 1e-4 for dL/dx
  and dL/dy (the central difference carries (eps/sigma)^2/6 ~ 2e-5);
* the exact solver's analytic gradient: within 10x the FMM's own relative
  error on the potential (5 nodes interpolate this Gaussian to ~2e-4);
* finite differences of the exact sum against the exact gradient
  (validates the grad f kernels), <= 1e-4 of the largest.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

N = 65536
EPS = 1e-3
DEPTH = 6
PO = 4


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


def _loss(ctx, X, Y, W, G):
    c, _ = ctx.solve(X, Y, W, poly_ord=PO, depth=DEPTH)
    return float(np.dot(G, c))


def test_adjoint_matches_fd_of_the_fmm(ctx, problem):
    _, dx, dy, dw = _grads(problem)
    dx, dy, dw = dx.cpu().numpy(), dy.cpu().numpy(), dw.cpu().numpy()
    x, y, w, g = problem
    X, Y, W, G = (t.detach().cpu().numpy().copy() for t in (x, y, w, g))
    ctx.set_kernel("gaussian", 0.01)
    tb0, sb0, _, _ = ctx.tree_export(X, Y, DEPTH)
    r = np.random.default_rng(9)
    res = {"dx": [], "dy": [], "dw": []}
    skipped = 0
    for i, q in zip(r.choice(N, 64, replace=False), r.integers(0, 3, 64)):
        # dL/dw_i: L is linear in w
        Wp, Wm = W.copy(), W.copy()
        Wp[i] += EPS
        Wm[i] -= EPS
        res["dw"].append((dw[i], (_loss(ctx, X, Y, Wp, G) - _loss(ctx, X, Y, Wm, G)) / (2 * EPS)))
        for name, arr, grad in (("dx", X, dx), ("dy", Y, dy)):
            Ap, Am = arr.copy(), arr.copy()
            Ap[i, q] += EPS
            Am[i, q] -= EPS
            same = True
            for A in (Ap, Am):
                tb, sb, _, _ = ctx.tree_export(A if name == "dx" else X, A if name == "dy" else Y, DEPTH)
                same &= (tb[i] == tb0[i]) if name == "dx" else (sb[i] == sb0[i])
            if not same:
                skipped += 1
                continue
            if name == "dx":
                lp, lm = _loss(ctx, Ap, Y, W, G), _loss(ctx, Am, Y, W, G)
            else:
                lp, lm = _loss(ctx, X, Ap, W, G), _loss(ctx, X, Am, W, G)
            res[name].append((grad[i, q], (lp - lm) / (2 * EPS)))
    assert skipped < 40
    for name, tol in (("dw", 1e-5), ("dx", 1e-4), ("dy", 1e-4)):
        a = np.array(res[name])
        err = np.max(np.abs(a[:, 0] - a[:, 1])) / np.max(np.abs(a[:, 1]))
        assert err <= tol, (name, err, len(a))


@pytest.mark.parametrize("precision", ["fp64", "tf32x3"])
def test_adjoint_close_to_exact_gradient(ctx, problem, precision):
    c, dx, dy, dw = _grads(problem, precision)
    x, y, w, g = problem
    X, Y, W, G = (t.detach() for t in (x, y, w, g))
    ctx.set_kernel("gaussian", 0.01)
    ce, cg, _ = ctx.solve_grad(X, Y, W, solver="exact")
    u, ug, _ = ctx.solve_grad(Y, X, G, solver="exact")
    e_pot = rel_l2(c.cpu().numpy(), ce.cpu().numpy())
    assert e_pot <= 1e-3
    for got, want, name in ((dx, G.unsqueeze(-1) * cg, "dx"), (dy, W.unsqueeze(-1) * ug, "dy"), (dw, u, "dw")):
        e = rel_l2(got.cpu().numpy(), want.cpu().numpy())
        assert e <= 10 * e_pot, (precision, name, e, e_pot)


def test_exact_gradient_matches_fd_of_exact_sum(ctx, problem):
    x, y, w, g = problem
    X, Y, W = (t.detach().cpu().numpy().copy() for t in (x, y, w))
    ctx.set_kernel("gaussian", 0.01)
    r = np.random.default_rng(10)
    rows = r.choice(N, 64, replace=False)
    _, cg, _ = ctx.solve_grad(X, Y, W, solver="exact")
    pairs = []
    for i, q in zip(rows, r.integers(0, 3, 64)):
        xp, xm = X.copy(), X.copy()
        xp[i, q] += EPS
        xm[i, q] -= EPS
        fd = (ctx.exact_rows([i], xp, Y, W)[0] - ctx.exact_rows([i], xm, Y, W)[0]) / (2 * EPS)
        pairs.append((cg[i, q], fd))
    a = np.array(pairs)
    assert np.max(np.abs(a[:, 0] - a[:, 1])) / np.max(np.abs(a[:, 1])) <= 1e-4
