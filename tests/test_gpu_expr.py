"""Kernels given as C++ expressions, compiled at run time (fmma_set_kernel_expr).

* an expression that restates a built-in kernel gives the built-in results
  (FP64 FMM and exact, <= 1e-12 rel-L2: same arithmetic up to operation order);
* a kernel that is not translation invariant (per-pair M2L path) matches a
  numpy direct sum through the exact solver (<= 1e-12) and the FMM matches the
  exact sum within its interpolation error;
* the mixed-precision sweep accepts an expression kernel;
* pyfmma's set_fn2 takes an expression string;
* a malformed expression is rejected when set, with the compiler's log.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _pts(d, n, seed):
    r = np.random.default_rng(seed)
    return r.random((n, d)), r.random((n, d)), r.standard_normal(n)


@pytest.mark.parametrize("d,builtin,p0,expr", [
    (3, "inv_r_safe", 0.0, "r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0"),
    (2, "gaussian", 0.01, "exp(-r2 / 0.01)"),
    (2, "multiquadric", 1e-4, "sqrt(r2 + 1e-4)"),
])
def test_expression_equals_builtin(ctx, d, builtin, p0, expr):
    import fmma_b200
    t, s, w = _pts(d, 12000, 31 + d)
    ctx.set_kernel(builtin, p0)
    want_fmm, _ = ctx.solve(t, s, w, poly_ord=5, depth=4)
    want_ex, _ = ctx.solve(t, s, w, solver="exact")
    c2 = fmma_b200.Context(0)
    try:
        c2.set_kernel_expr(expr, translation_invariant=True)
        got_fmm, _ = c2.solve(t, s, w, poly_ord=5, depth=4)
        got_ex, _ = c2.solve(t, s, w, solver="exact")
    finally:
        c2.close()
    assert rel_l2(got_ex, want_ex) <= 1e-12
    assert rel_l2(got_fmm, want_fmm) <= 1e-12


def test_general_kernel_against_numpy_and_exact():
    import fmma_b200
    d = 2
    t, s, w = _pts(d, 3000, 7)
    expr = "1.0 / (1.0 + x[0] * x[0] + y[1] * y[1] + r2)"
    c = fmma_b200.Context(0)
    try:
        c.set_kernel_expr(expr, translation_invariant=False)
        ex, _ = c.solve(t, s, w, solver="exact")
        fm, _ = c.solve(t, s, w, poly_ord=7, depth=4)
    finally:
        c.close()
    sub = slice(0, 400)
    K = 1.0 / (1.0 + t[sub, 0:1] ** 2 + (s[:, 1] ** 2)[None, :]
               + ((t[sub, None, :] - s[None, :, :]) ** 2).sum(-1))
    assert rel_l2(ex[sub], K @ w) <= 1e-12
    assert rel_l2(fm, ex) <= 1e-6


def test_expression_kernel_mixed_precision():
    import fmma_b200
    t, s, w = _pts(3, 30000, 11)
    c = fmma_b200.Context(0)
    try:
        c.set_kernel_expr("r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0", translation_invariant=True)
        plain, _ = c.solve(t, s, w, poly_ord=5, depth=5)
        mixed, _ = c.solve(t, s, w, poly_ord=5, depth=5, precision="tf32x3")
    finally:
        c.close()
    assert rel_l2(mixed, plain) <= 2e-5


def test_pyfmma_set_fn2_accepts_expression():
    import pyfmma
    t, s, w = _pts(2, 5000, 13)
    a = pyfmma.fmmad2()
    a.set_solver_type("fmm")
    a.set_poly_ord(4)
    a.set_fn2(pyfmma.kernels.gaussian(0.01))
    want = np.zeros(len(t))
    a.solve(t, w, s, want)
    b = pyfmma.fmmad2()
    b.set_solver_type("fmm")
    b.set_poly_ord(4)
    b.set_fn2("exp(-r2 / 0.01)")
    got = np.zeros(len(t))
    b.solve(t, w, s, got)
    assert rel_l2(got, want) <= 1e-12


def test_malformed_expression_is_rejected():
    import fmma_b200
    c = fmma_b200.Context(0)
    try:
        with pytest.raises(fmma_b200.FmmaError) as ei:
            c.set_kernel_expr("exp(-r2 / ", translation_invariant=True)
        assert "does not compile" in str(ei.value)
    finally:
        c.close()
