"""Forests of independent problems in one sweep (the C5 shape, reduced):
every problem's result equals the single-problem solve of that problem.

Tolerances: plain FP64 forest vs single solves, relative L2 <= 1e-13 per
problem (same kernels, same per-row summation order); mixed forest vs
single mixed solves <= 2e-6: on levels with fewer 128-row tiles than SMs the
tensor-core M2L splits each tile's far slots over several CTAs, so a lone
problem and the same problem inside a forest sum their FP32 partial
products in different groupings (differences at the FP32 rounding level,
well below the FMM's own truncation error); FP64 forest vs the FP64 exact
sum within the FMM's own truncation error."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _forest(nprob, seed, lo=300, hi=6000, R=3, d=2):
    r = np.random.default_rng(seed)
    sizes = np.exp(r.uniform(np.log(lo), np.log(hi), nprob)).astype(int)
    sizes[0] = 40  # a problem whose Depth stays below 3 (no far field)
    tg, sr = [], []
    for m in sizes:
        side = r.uniform(0.5, 2.0)
        corner = r.uniform(-3, 3, d)
        tg.append(corner + side * r.random((m, d)))
        sr.append(corner + side * r.random((m, d)))
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    W = r.standard_normal((R, off[-1]))
    return np.concatenate(tg), off, np.concatenate(sr), off.copy(), W, sizes


@pytest.mark.parametrize("precision", ["fp64", "tf32x3"])
def test_forest_equals_single_solves(ctx, precision):
    tgt, toff, src, soff, W, sizes = _forest(24, 1)
    ctx.set_kernel("multiquadric", 1e-4)
    depths = ctx.forest_depths(tgt, toff, src, soff, 32)
    assert depths.min() <= 2 and depths.max() >= 5
    out = ctx.forest_solve(tgt, toff, src, soff, W, depths, poly_ord=4, precision=precision)
    assert out.shape == (3, toff[-1])
    tol = 1e-13 if precision == "fp64" else 2e-6
    for p in range(len(sizes)):
        t = np.ascontiguousarray(tgt[toff[p]:toff[p + 1]])
        s = np.ascontiguousarray(src[soff[p]:soff[p + 1]])
        w = np.ascontiguousarray(W[:, soff[p]:soff[p + 1]])
        one, _ = ctx.solve(t, s, w, poly_ord=4, depth=int(depths[p]), precision=precision)
        assert rel_l2(out[:, toff[p]:toff[p + 1]], one) <= tol, (p, depths[p])


def test_forest_against_exact(ctx):
    tgt, toff, src, soff, W, sizes = _forest(16, 2, R=1)
    ctx.set_kernel("log_r")
    depths = ctx.forest_depths(tgt, toff, src, soff, 32)
    out = ctx.forest_solve(tgt, toff, src, soff, W[0], depths, poly_ord=5)
    for p in (0, 5, 15):
        t = np.ascontiguousarray(tgt[toff[p]:toff[p + 1]])
        s = np.ascontiguousarray(src[soff[p]:soff[p + 1]])
        ex, _ = ctx.solve(t, s, np.ascontiguousarray(W[0, soff[p]:soff[p + 1]]), solver="exact")
        assert rel_l2(out[toff[p]:toff[p + 1]], ex) <= 1e-4


def test_forest_of_one_is_a_solve(ctx, oracle):
    r = np.random.default_rng(3)
    t, s, w = r.random((5000, 3)), r.random((5000, 3)), r.uniform(-1, 1, 5000)
    ctx.set_kernel("inv_r_safe")
    out = ctx.forest_solve(t, [0, 5000], s, [0, 5000], w, [5], poly_ord=4)
    ref, _ = oracle.fmm(3, 1, 0.0, 4, 5, 0, t, s, w)
    assert rel_l2(out, ref) <= 1e-12


def test_plan_replays_graph_and_matches_forest_solve(ctx):
    tgt, toff, src, soff, W, sizes = _forest(20, 5, R=4)
    ctx.set_kernel("multiquadric", 1e-4)
    depths = ctx.forest_depths(tgt, toff, src, soff, 32)
    plan = ctx.plan(tgt, toff, src, soff, 4, depths, poly_ord=4, precision="fp64")
    st = plan.stats()
    assert st["graph_nodes"] > 10 and st["levels_fp64"] >= 1
    want = ctx.forest_solve(tgt, toff, src, soff, W, depths, poly_ord=4)
    got = plan.execute(W)
    assert np.array_equal(got, want)
    # a second weight set through the same graph
    W2 = np.random.default_rng(6).standard_normal(W.shape)
    assert np.array_equal(plan.execute(W2), ctx.forest_solve(tgt, toff, src, soff, W2, depths, poly_ord=4))
    plan.close()


def test_plan_autotunes_mixed_levels(ctx, tmp_path):
    tgt, toff, src, soff, W, sizes = _forest(20, 7, R=4)
    ctx.set_kernel("multiquadric", 1e-4)
    depths = ctx.forest_depths(tgt, toff, src, soff, 32)
    path = str(tmp_path / "tuner.txt")
    ctx.set_tuner_cache(path)
    plan = ctx.plan(tgt, toff, src, soff, 4, depths, poly_ord=4, precision="bf16x3", autotune=True)
    st = plan.stats()
    assert st["levels_tc"] + st["levels_fp64"] >= 3
    got = plan.execute(W)
    plain = ctx.forest_solve(tgt, toff, src, soff, W, depths, poly_ord=4)
    assert rel_l2(got, plain) <= 2e-5
    plan.close()
    import os
    assert os.path.getsize(path) > 0
    # per level FP64 DMMA (0) or the tensor-core kernel, 1-SM or 2-SM with 1, 2 or 4 units
    # per pipeline stage (1 + 2 i + pair); per level the slot split (0-3); for the
    # leaves the L2P layout (1 lanes over targets, 2 over coefficients)
    entries = dict(line.split() for line in open(path) if line.strip())
    engines = [int(v) for k, v in entries.items() if k.startswith("m2l")]
    splits = [int(v) for k, v in entries.items() if k.startswith("split_")]
    leaves = [int(v) for k, v in entries.items() if k.startswith("l2p")]
    assert engines and set(engines) <= set(range(7)), engines
    assert len(splits) == len(engines) and set(splits) <= {0, 1, 2, 3}, splits
    assert leaves and set(leaves) <= {1, 2}, leaves


def test_plan_engines_agree_on_a_large_level(ctx):
    """A single 3-D problem whose leaf level has enough 256-row tiles for the
    2-SM kernel: the plan (autotuned engines per level, graph replay) agrees
    with the direct mixed solve to FP32 rounding and with plain FP64 to 1e-5."""
    r = np.random.default_rng(61)
    n = 300000
    t, s, w = r.random((n, 3)), r.random((n, 3)), r.uniform(-1, 1, n)
    ctx.set_kernel("inv_r_safe")
    plan = ctx.plan(t, [0, n], s, [0, n], 1, [6], poly_ord=5, precision="bf16x3", autotune=True)
    got = plan.execute(w)
    plan.close()
    direct, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision="bf16x3")
    plain, _ = ctx.solve(t, s, w, poly_ord=5, depth=6)
    assert rel_l2(got, direct) <= 1e-6, rel_l2(got, direct)
    assert rel_l2(got, plain) <= 1e-5
