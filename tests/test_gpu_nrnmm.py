"""The nrnmm solver (src/nrnmm.cpp:13-102: one grid of nrn_N^d boxes, P2M,
M2P from every box not adjacent to the target's, P2P from the adjacent ones)
on the GPU:

* against the compiled reference's outputs (golden vectors, the reference's
  own test kernels and orders among them): FP64 inputs within 1e-12 relative
  L2 (only the order of the sums differs), FP32 inputs within 1e-5 (the
  reference computes in float, the GPU path in double after binning in float);
* against the C oracle on a larger seeded case;
* nrn_N 1 and 2 (every box adjacent) equal the exact sum;
* multi-RHS equals single solves; an expression kernel (far field through the
  hook) equals the built-in kernel; pyfmma's solver type "nrnmm" keeps the
  reference's sticky default nrn_N;
* at 200k points, where the oracle is too slow: linearity in the weights and
  the error against exact sums at sampled targets.
"""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu

CASES = ["nrnmm_inv_r_d1", "nrnmm_inv_r_d2_f32", "nrnmm_sum_r2_d2", "nrnmm_sum2_r2_d2", "nrnmm_inv_diff_d1",
         "nrnmm_inv_r_safe_d3", "nrnmm_gaussian_d2_default_nrn", "nrnmm_log_r_d2_f32", "nrnmm_clustered_d3"]


@pytest.mark.parametrize("name", CASES)
def test_nrnmm_matches_reference(ctx, name):
    g = golden(name)
    ctx.set_kernel(int(g["kernel"]), float(g["p0"]))
    w = g["w"] if "w" in g else None
    got, used = ctx.solve(g["tgt"], g["src"], w, solver="nrnmm", poly_ord=int(g["poly_ord"]), depth=int(g["nrn"]))
    assert used == int(g["nrn_used"])
    assert got.dtype == g["tgt"].dtype
    tol = 1e-5 if g["tgt"].dtype == np.float32 else 1e-12
    assert rel_l2(got, g["nrnmm"]) <= tol


@pytest.mark.parametrize("d,kid,p0,po", [(3, 1, 0.0, 4), (2, 5, 1e-3, 5)])
def test_nrnmm_matches_oracle(ctx, oracle, d, kid, p0, po):
    r = np.random.default_rng(21 + d)
    t, s, w = r.random((8000, d)), r.random((7000, d)), r.standard_normal(7000)
    ctx.set_kernel(kid, p0)
    got, used = ctx.solve(t, s, w, solver="nrnmm", poly_ord=po, depth=-1)
    want, used_o = oracle.nrnmm(d, kid, p0, po, -1, t, s, w)
    assert used == used_o
    assert rel_l2(got, want) <= 1e-12


@pytest.mark.parametrize("nrn", [1, 2])
def test_nrnmm_small_grid_is_exact(ctx, nrn):
    r = np.random.default_rng(nrn)
    t, s, w = r.random((3000, 2)), r.random((2500, 2)), r.standard_normal(2500)
    ctx.set_kernel("inv_r_safe")
    got, _ = ctx.solve(t, s, w, solver="nrnmm", poly_ord=3, depth=nrn)
    ex, _ = ctx.solve(t, s, w, solver="exact")
    assert rel_l2(got, ex) <= 1e-13


def test_nrnmm_multi_rhs_equals_single(ctx):
    r = np.random.default_rng(5)
    t, s = r.random((4000, 3)), r.random((3000, 3))
    W = r.standard_normal((6, 3000))
    ctx.set_kernel("inv_r_safe")
    out, _ = ctx.solve(t, s, W, solver="nrnmm", poly_ord=3, depth=6)
    for k in range(6):
        one, _ = ctx.solve(t, s, W[k], solver="nrnmm", poly_ord=3, depth=6)
        assert rel_l2(out[k], one) <= 1e-14


def test_nrnmm_expression_kernel_equals_builtin(ctx):
    import fmma_b200
    r = np.random.default_rng(8)
    t, s, w = r.random((5000, 2)), r.random((5000, 2)), r.standard_normal(5000)
    ctx.set_kernel("gaussian", 0.01)
    want, _ = ctx.solve(t, s, w, solver="nrnmm", poly_ord=5, depth=9)
    c2 = fmma_b200.Context(0)
    try:
        c2.set_kernel_expr("exp(-r2 / 0.01)", translation_invariant=True)
        got, used = c2.solve(t, s, w, solver="nrnmm", poly_ord=5, depth=9)
    finally:
        c2.close()
    assert used == 9
    assert rel_l2(got, want) <= 1e-12


def test_pyfmma_nrnmm_sticky_default_grid():
    import pyfmma
    g = golden("nrnmm_gaussian_d2_default_nrn")
    f = pyfmma.fmmad2()
    f.set_solver_type("nrnmm")
    f.set_poly_ord(int(g["poly_ord"]))
    f.set_fn2(pyfmma.kernels.gaussian(float(g["p0"])))
    ans = np.zeros(len(g["tgt"]))
    f.solve(g["tgt"], g["w"], g["src"], ans)
    assert rel_l2(ans, g["nrnmm"]) <= 1e-12
    assert f._nrn_N == int(g["nrn_used"])


def test_nrnmm_large_linearity_and_error(ctx):
    r = np.random.default_rng(13)
    n = 200_000
    t, s = r.random((n, 2)), r.random((n, 2))
    w1, w2 = r.standard_normal(n), r.standard_normal(n)
    ctx.set_kernel("inv_r_safe")
    a1, used = ctx.solve(t, s, w1, solver="nrnmm", poly_ord=5, depth=-1)
    a2, _ = ctx.solve(t, s, w2, solver="nrnmm", poly_ord=5, depth=-1)
    a12, _ = ctx.solve(t, s, w1 + w2, solver="nrnmm", poly_ord=5, depth=-1)
    assert used == int(np.sqrt(3.0) * n ** 0.25) + 1
    assert rel_l2(a12, a1 + a2) <= 1e-13
    rows = r.choice(n, 2000, replace=False)
    ex = ctx.exact_rows(rows, t, s, w1)
    assert rel_l2(a1[rows], ex) <= 1e-5
