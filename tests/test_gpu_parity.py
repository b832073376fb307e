"""GPU parity: the plain FP64 fmm and the exact solver through the C ABI
against the reference's own outputs (golden vectors) and the oracle.

Tolerances: plain FP64 fmm vs the reference fmm, relative L2 <= 1e-12 and
max |diff| <= 1e-11 * max|ref| (summation order differs, nothing else);
exact vs exact, relative L2 <= 1e-13."""
import numpy as np
import pytest

from conftest import golden, golden_names, rel_l2, rel_rms

pytestmark = pytest.mark.gpu

FMM_CASES = [n for n in golden_names() if not n.startswith(("bins", "f", "tree", "nrnmm", "cheb"))]
TOL = 1e-12


def _solve(ctx, g, solver="fmm", precision="fp64", depth=None, w=True):
    ctx.set_kernel(int(g["kernel"]), float(g["p0"]))
    ww = g.get("w") if w else None
    return ctx.solve(g["tgt"], g["src"], ww, solver=solver, poly_ord=int(g["poly_ord"]),
                     depth=int(g["depth"]) if depth is None else depth, trans_sym=int(g["trans_sym"]),
                     precision=precision)


@pytest.mark.parametrize("name", FMM_CASES)
def test_fmm_fp64_matches_reference(ctx, name):
    g = golden(name)
    out, used = _solve(ctx, g)
    assert used == int(g["depth_used"])
    ref = g["fmm"]
    assert rel_l2(out, ref) <= TOL, rel_l2(out, ref)
    assert np.max(np.abs(out - ref)) <= 10 * TOL * np.max(np.abs(ref))


@pytest.mark.parametrize("name", [n for n in FMM_CASES if "default" not in n and "L7" not in n])
def test_exact_matches_reference(ctx, name):
    g = golden(name)
    if "exact" not in g:
        pytest.skip("no exact vector")
    out, _ = _solve(ctx, g, solver="exact")
    assert rel_l2(out, g["exact"]) <= 1e-13


def test_float_instantiation_matches_reference(ctx):
    g = golden("f2_log_r_n5_L5")
    out, _ = _solve(ctx, g)
    assert out.dtype == np.float32
    # the reference computes in float; this build computes in FP64 with the
    # reference's float binning, so the two differ by float rounding only
    assert rel_l2(out, g["fmm"]) <= 2e-5
    e, _ = _solve(ctx, g, solver="exact")
    assert rel_l2(e, g["exact"]) <= 2e-6


@pytest.mark.parametrize("d,kid,po,depth,ts,n", [
    (1, 2, 7, 9, 0, 5000), (1, 3, 4, 10, 1, 20000), (2, 3, 5, 7, 0, 30000), (2, 5, 4, 6, 1, 20000),
    (3, 1, 5, 5, 1, 20000), (3, 4, 4, 4, 0, 10000), (3, 1, 2, 6, 0, 30000), (2, 6, 3, 6, 1, 10000),
    # sparse leaves (fewer than 16 targets a leaf): the fused leaf L2L+L2P, down to Depth 3
    (3, 1, 6, 3, 0, 4000), (2, 3, 7, 3, 1, 600), (2, 5, 7, 5, 0, 6000), (3, 4, 3, 4, 1, 8000),
])
def test_fmm_fp64_matches_oracle_random(ctx, oracle, d, kid, po, depth, ts, n):
    r = np.random.default_rng(77 + d * 10 + kid)
    t, s, w = r.random((n, d)), r.random((n, d)), r.uniform(-1, 1, n)
    p0 = 1e-4 if kid == 5 else 0.01
    ctx.set_kernel(kid, p0)
    out, _ = ctx.solve(t, s, w, solver="fmm", poly_ord=po, depth=depth, trans_sym=ts)
    ref, _ = oracle.fmm(d, kid, p0, po, depth, ts, t, s, w)
    assert rel_l2(out, ref) <= TOL


def test_multi_rhs_equals_single_solves(ctx):
    r = np.random.default_rng(3)
    t, s = r.random((4000, 2)), r.random((5000, 2))
    W = r.standard_normal((5, 5000))
    ctx.set_kernel("log_r")
    out, _ = ctx.solve(t, s, W, poly_ord=4, depth=5)
    assert out.shape == (5, 4000)
    for k in range(5):
        one, _ = ctx.solve(t, s, np.ascontiguousarray(W[k]), poly_ord=4, depth=5)
        assert rel_l2(out[k], one) <= 1e-14


@pytest.mark.parametrize("nrhs", [3, 9, 12, 17])
def test_multi_rhs_staged_l2p_matches_oracle(ctx, oracle, nrhs):
    # 2-D, 4 nodes/dim (16 coefficients) and ~90 targets a leaf: the target-lane
    # L2P with the leaf's local expansion staged in shared memory, whose last
    # rhs pass reads a whole block of 8 (R % 8 = 1..4 for 9, 12, 17)
    r = np.random.default_rng(12 + nrhs)
    t, s = r.random((6000, 2)), r.random((5000, 2))
    W = r.standard_normal((nrhs, 5000))
    ctx.set_kernel("log_r")
    out, _ = ctx.solve(t, s, W, poly_ord=3, depth=4)
    for k in range(nrhs):
        ref, _ = oracle.fmm(2, 3, 0.0, 3, 4, 0, t, s, np.ascontiguousarray(W[k]))
        assert rel_l2(out[k], ref) <= TOL, (k, rel_l2(out[k], ref))


def test_unweighted_equals_unit_weights(ctx):
    r = np.random.default_rng(4)
    t, s = r.random((3000, 3)), r.random((3000, 3))
    ctx.set_kernel("inv_r_safe")
    a, _ = ctx.solve(t, s, None, poly_ord=3, depth=4)
    b, _ = ctx.solve(t, s, np.ones(3000), poly_ord=3, depth=4)
    assert np.array_equal(a, b)


def test_empty_and_tiny_inputs(ctx):
    ctx.set_kernel("inv_r_safe")
    t = np.random.default_rng(5).random((10, 3))
    out, _ = ctx.solve(t, np.zeros((0, 3)), np.zeros(0), poly_ord=3, depth=4)
    assert np.all(out == 0)
    out, _ = ctx.solve(np.zeros((0, 3)), t, np.ones(10), poly_ord=3, depth=4)
    assert out.shape == (0,)
    # one target, one source, depth 1 (P2P only)
    out, _ = ctx.solve(t[:1], t[1:2], np.ones(1), poly_ord=2, depth=1)
    assert abs(out[0] - 1.0 / np.linalg.norm(t[0] - t[1])) < 1e-14
    # coincident target and source: 0 for the guarded kernel
    out, _ = ctx.solve(t[:3], t[:3], np.ones(3), poly_ord=2, depth=2)
    e = sum(1.0 / np.linalg.norm(t[0] - t[j]) for j in (1, 2))
    assert abs(out[0] - e) < 1e-12 * e


def test_depth_default_is_reference_rule(ctx, oracle):
    r = np.random.default_rng(6)
    t, s = r.random((3000, 2)), r.random((3000, 2))
    ctx.set_kernel("log_r")
    out, used = ctx.solve(t, s, None, poly_ord=3, depth=-1)
    assert used == oracle.default_depth(3000, 2)
    ref, _ = oracle.fmm(2, 3, 0.0, 3, -1, 0, t, s, None)
    assert rel_l2(out, ref) <= TOL


def test_nonfinite_coordinates_rejected(ctx):
    import fmma_b200
    t = np.random.default_rng(7).random((100, 2))
    t[5, 1] = np.nan
    ctx.set_kernel("log_r")
    with pytest.raises(fmma_b200.FmmaError) as e:
        ctx.solve(t, t.copy(), None, poly_ord=3, depth=4)
    assert e.value.status == 1


def test_device_pointers_match_host(ctx):
    import torch
    r = np.random.default_rng(8)
    t, s, w = r.random((20000, 3)), r.random((20000, 3)), r.standard_normal(20000)
    ctx.set_kernel("inv_r_safe")
    host, _ = ctx.solve(t, s, w, poly_ord=4, depth=5)
    dev, _ = ctx.solve(torch.from_numpy(t).cuda(), torch.from_numpy(s).cuda(), torch.from_numpy(w).cuda(),
                       poly_ord=4, depth=5)
    assert np.array_equal(host, dev.cpu().numpy())


def test_repeat_solves_are_deterministic(ctx):
    r = np.random.default_rng(9)
    t, s, w = r.random((30000, 2)), r.random((30000, 2)), r.standard_normal(30000)
    ctx.set_kernel("log_r")
    a, _ = ctx.solve(t, s, w, poly_ord=5, depth=7)
    b, _ = ctx.solve(t, s, w, poly_ord=5, depth=7)
    assert np.array_equal(a, b)


def test_exact_rows_sampled_oracle(ctx, oracle):
    r = np.random.default_rng(10)
    t, s, w = r.random((5000, 3)), r.random((6000, 3)), r.standard_normal(6000)
    rows = r.choice(5000, 300, replace=False)
    ctx.set_kernel("inv_r_safe")
    got = ctx.exact_rows(rows, t, s, w)
    want = oracle.exact_rows(3, 1, 0.0, rows, t, s, w)
    assert rel_l2(got, want) <= 1e-13


@pytest.mark.parametrize("d,po", [(1, 3), (2, 3), (2, 4)])
def test_reference_accuracy_contract(ctx, d, po):
    # test/src/fmma/fmm.cpp:10-61 and common.cpp: fmm rel-RMS vs exact < 1e-3
    r = np.random.default_rng(11 + d)
    t, s = r.random((20, d)) - 0.5, r.random((10, d)) - 0.5
    ctx.set_kernel("inv_r")
    a, _ = ctx.solve(t, s, None, poly_ord=po, depth=3)
    e, _ = ctx.solve(t, s, None, solver="exact")
    assert rel_rms(a, e) < 1e-3
