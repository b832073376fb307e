"""The global Chebyshev approximation (CHEBYSHEV_APPROX, src/chebyshev_approx.cpp:
36-101) on the GPU:

* fit: the coefficients from the node values equal the C oracle's direct
  solve of the reference's collocation system within 1e-12 (relative L2); the
  reference's own coefficients (GCR stopped at a squared residual of 1e-6) lie
  within 1e-3 of them;
* evaluation: with the reference's coefficients, the GPU predictions equal
  the compiled reference's predict within 1e-13 relative L2 (Clenshaw against
  cos(k acos x) products);
* the reference's tests (test/src/chebyshev_approx/common.cpp): T_n T_m gives
  the unit coefficient vector, smooth functions are predicted within 1e-6;
* several functions in one call equal single calls; device (torch) arrays;
  a point outside [-1, 1] is rejected.
"""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu

CASES = ["cheb_t2_d1", "cheb_t1t3_d2", "cheb_exp_cos_d1", "cheb_inv1p_d2", "cheb_inv1p_d3", "cheb_len2_d3",
         "cheb_exp_cos_d2"]


@pytest.mark.parametrize("name", CASES)
def test_cheb_fit_matches_oracle_and_reference(ctx, oracle, name):
    g = golden(name)
    dim, nth = int(g["dim"]), int(g["nth"])
    got = ctx.cheb_fit(g["values"], dim, nth)
    want = oracle.cheb_fit(dim, nth, g["values"])
    assert rel_l2(got, want) <= 1e-12 or np.linalg.norm(got - want) <= 1e-14
    assert np.linalg.norm(got - g["coef"]) <= 1e-3


@pytest.mark.parametrize("name", CASES)
def test_cheb_eval_matches_reference(ctx, name):
    g = golden(name)
    got = ctx.cheb_eval(g["coef"], g["pts"], int(g["nth"]))
    assert rel_l2(got, g["predict"]) <= 1e-13


def test_cheb_reference_tests():
    """test/src/chebyshev_approx/common.cpp: coef tests (T_n(x), T_n(x) T_m(y),
    Nth 10 / 5) and predict tests (tolerance 1e-6 on the squared error)."""
    import fmma_b200
    ctx = fmma_b200.default_context(0)
    T = [lambda v: np.ones_like(v), lambda v: v, lambda v: 2 * v * v - 1, lambda v: 4 * v ** 3 - 3 * v]
    for n in range(4):
        P = fmma_b200.cheb_points(1, 10)
        c = ctx.cheb_fit(T[n](P[:, 0]), 1, 10)
        e = np.zeros(11)
        e[n] = 1.0
        assert np.sum((c - e) ** 2) < 1e-20
    for n, m in [(0, 0), (0, 1), (2, 0), (1, 3)]:
        P = fmma_b200.cheb_points(2, 5)
        c = ctx.cheb_fit(T[n](P[:, 0]) * T[m](P[:, 1]), 2, 5)
        e = np.zeros(36)
        e[m * 6 + n] = 1.0
        assert np.sum((c - e) ** 2) < 1e-20
    r = np.random.default_rng(0)
    for dim, nth, f in [(1, 10, lambda p: np.exp(p[:, 0])),
                        (2, 10, lambda p: np.cos(p[:, 0]) * np.sin(p[:, 1])),
                        (3, 12, lambda p: 1.0 / (1.0 + np.sum(p * p, axis=1)))]:
        c = ctx.cheb_fit(f(fmma_b200.cheb_points(dim, nth)), dim, nth)
        x = r.uniform(-1, 1, (10, dim))
        assert np.sum((ctx.cheb_eval(c, x, nth) - f(x)) ** 2) < 1e-6


def test_cheb_batched_and_device_arrays(ctx):
    import torch
    import fmma_b200
    r = np.random.default_rng(3)
    dim, nth = 3, 7
    V = r.standard_normal((4, (nth + 1) ** dim))
    C = ctx.cheb_fit(V, dim, nth)
    pts = r.uniform(-1, 1, (5000, dim))
    E = ctx.cheb_eval(C, pts, nth)
    for f in range(4):
        assert np.array_equal(ctx.cheb_fit(V[f], dim, nth), C[f])
        assert np.array_equal(ctx.cheb_eval(C[f], pts, nth), E[f])
    Cd = ctx.cheb_fit(torch.from_numpy(V).cuda(), dim, nth)
    Ed = ctx.cheb_eval(Cd, torch.from_numpy(pts).cuda(), nth)
    assert np.array_equal(Cd.cpu().numpy(), C) and np.array_equal(Ed.cpu().numpy(), E)
    # the fit interpolates: predictions at the nodes give the values back
    back = ctx.cheb_eval(C, fmma_b200.cheb_points(dim, nth), nth)
    assert np.max(np.abs(back - V)) <= 1e-12


def test_cheb_eval_rejects_points_outside(ctx):
    import fmma_b200
    c = np.zeros(36)
    with pytest.raises(fmma_b200.FmmaError) as ei:
        ctx.cheb_eval(c, np.array([[0.5, 1.5]]), 5)
    assert ei.value.status == 1
