"""Mixed precision on the GPU: tcgen05 split-precision M2L (TF32x3 / BF16x3)
and FP32 P2P with two-sum compensated accumulation, against the plain FP64
FMM and the FP64 exact sum.

Tolerances: against the FP64 exact sum the mixed error stays within 2x the
plain FMM's.  Mixed and plain agree to relative L2
<= 1e-5: split products carry ~2^-21 (TF32x3) / ~2^-17 (BF16x3) relative
error, and the tensor-core FP32 accumulation (round toward zero) is drained
into FP32 registers every few slots."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(d, n, seed, clustered=False):
    r = np.random.default_rng(seed)
    if clustered:
        c = r.uniform(0.2, 0.8, (6, d))
        t = np.clip(c[r.integers(0, 6, n)] + 0.03 * r.standard_normal((n, d)), 0, 1)
        s = np.clip(c[r.integers(0, 6, n)] + 0.03 * r.standard_normal((n, d)), 0, 1)
    else:
        t, s = r.random((n, d)), r.random((n, d))
    return t, s, r.uniform(-1, 1, n)


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3"])
@pytest.mark.parametrize("d,kern,po,depth,n,clustered", [
    (3, "inv_r_safe", 5, 5, 40000, False),
    (3, "inv_r_safe", 5, 6, 60000, True),
    (2, "log_r", 5, 7, 100000, False),
    (3, "gaussian", 4, 5, 40000, False),
    (2, "multiquadric", 4, 6, 40000, False),
])
def test_mixed_matches_plain_and_exact(ctx, prec, d, kern, po, depth, n, clustered):
    t, s, w = _case(d, n, 100 + d, clustered)
    ctx.set_kernel(kern, 0.01 if kern == "gaussian" else 1e-4)
    plain, _ = ctx.solve(t, s, w, poly_ord=po, depth=depth, precision="fp64")
    mixed, _ = ctx.solve(t, s, w, poly_ord=po, depth=depth, precision=prec)
    assert rel_l2(mixed, plain) <= 1e-5, rel_l2(mixed, plain)
    rows = np.random.default_rng(1).choice(n, min(n, 2048), replace=False)
    ex = ctx.exact_rows(rows, t, s, w)
    e_plain, e_mixed = rel_l2(plain[rows], ex), rel_l2(mixed[rows], ex)
    if prec == "tf32x3" or d == 3:
        assert e_mixed <= 2.0 * e_plain + 1e-12, (e_mixed, e_plain)
    else:
        # BF16x3 products carry ~2^-17 relative error: where the plain FMM is
        # more accurate than that (low-order 2-D kernels) the bar is absolute
        assert e_mixed <= 1e-5, (e_mixed, e_plain)


@pytest.mark.parametrize("d,kern,po,depth,n", [(3, "inv_r_safe", 5, 5, 40000), (2, "log_r", 4, 6, 50000)])
def test_bf16x3_close_to_plain(ctx, d, kern, po, depth, n):
    t, s, w = _case(d, n, 200 + d)
    ctx.set_kernel(kern)
    plain, _ = ctx.solve(t, s, w, poly_ord=po, depth=depth, precision="fp64")
    mixed, _ = ctx.solve(t, s, w, poly_ord=po, depth=depth, precision="bf16x3")
    assert rel_l2(mixed, plain) <= 2e-5, rel_l2(mixed, plain)
    rows = np.random.default_rng(2).choice(n, 2048, replace=False)
    ex = ctx.exact_rows(rows, t, s, w)
    assert rel_l2(mixed[rows], ex) <= 2.0 * rel_l2(plain[rows], ex)


def test_mixed_multi_rhs_equals_single(ctx):
    """Four right-hand sides at once against one at a time.  The batch has
    four times the M2L rows, so levels that the tensor-core M2L splits over
    CTAs (fewer 128-row tiles than SMs) group the FP32 partial sums
    differently: agreement to the FP32 accumulation level, 5e-6."""
    t, s, _ = _case(3, 30000, 7)
    W = np.random.default_rng(8).standard_normal((4, 30000))
    ctx.set_kernel("inv_r_safe")
    out, _ = ctx.solve(t, s, W, poly_ord=4, depth=5, precision="tf32x3")
    for k in range(4):
        one, _ = ctx.solve(t, s, np.ascontiguousarray(W[k]), poly_ord=4, depth=5, precision="tf32x3")
        assert rel_l2(out[k], one) <= 5e-6


@pytest.mark.parametrize("R,depth", [(16, 5), (11, 7)])
def test_mixed_many_rhs_equals_single(ctx, R, depth):
    """9 to 16 right-hand sides take the 16-wide block of the mixed near field
    (two targets a lane; leaves of ~230 and ~15 targets); one at a time they
    take the 1-wide block.  Same FP32 regrouping bound as above."""
    r = np.random.default_rng(21)
    n = 60000
    t, s = r.random((n, 2)), r.random((n, 2))
    W = r.standard_normal((R, n))
    ctx.set_kernel("multiquadric", 1e-4)
    out, _ = ctx.solve(t, s, W, poly_ord=4, depth=depth, precision="tf32x3")
    for k in (0, R // 2, R - 1):
        one, _ = ctx.solve(t, s, np.ascontiguousarray(W[k]), poly_ord=4, depth=depth, precision="tf32x3")
        assert rel_l2(out[k], one) <= 5e-6, (k, rel_l2(out[k], one))


def test_mixed_is_deterministic(ctx):
    t, s, w = _case(3, 50000, 9, clustered=True)
    ctx.set_kernel("inv_r_safe")
    a, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision="tf32x3")
    b, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision="tf32x3")
    assert np.array_equal(a, b)


def test_mixed_non_translation_invariant_kernel_uses_fp64_path(ctx):
    t, s, w = _case(2, 3000, 10)
    ctx.set_kernel("sum2_over_r2")
    plain, _ = ctx.solve(t * 5 - 2.5, s * 5 - 2.5, w, poly_ord=3, depth=4, precision="fp64")
    mixed, _ = ctx.solve(t * 5 - 2.5, s * 5 - 2.5, w, poly_ord=3, depth=4, precision="tf32x3")
    assert np.array_equal(plain, mixed)


def test_mixed_1d_near_coincident_points(ctx):
    # 1/(x-y) with 4096 + 4096 uniform points: the closest pairs are ~1e-8
    # apart, far below the leaf width.  The double-float P2P keeps FP32
    # relative accuracy per term (the plain 1-D FMM is at ~1e-9 here, so the
    # mixed path is held to FP32-level accuracy, not to 2x plain).
    t = np.random.default_rng(1).random((4096, 1))
    s = np.random.default_rng(2).random((4096, 1))
    w = np.random.default_rng(3).uniform(-1, 1, 4096)
    ctx.set_kernel("inv_diff")
    plain, _ = ctx.solve(t, s, w, poly_ord=7, depth=8, precision="fp64")
    for prec in ("tf32x3", "bf16x3"):
        mixed, _ = ctx.solve(t, s, w, poly_ord=7, depth=8, precision=prec)
        assert rel_l2(mixed, plain) <= 2e-6, (prec, rel_l2(mixed, plain))


def _clusters(n, seed, k=16, sigma=0.02):
    """Points from k isotropic Gaussians (centres in [0.1, 0.9]^3), clipped to the cube."""
    r = np.random.default_rng(seed)
    c = r.uniform(0.1, 0.9, (k, 3))
    return np.clip(c[r.integers(0, k, n)] + sigma * r.standard_normal((n, 3)), 0, 1)


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3"])
def test_compensated_p2p_all_near(ctx, prec):
    """Depth 2: every leaf is a near neighbour of every other and there is no
    far field, so the whole result is the FP32 near field.  Each target lane
    sums the ~4,000 sources of a leaf in FP32: a plain FP32 running sum would
    carry ~u sqrt(n) ~ 4e-6 relative error here; with two-sum compensation
    only the FP32 kernel evaluations remain (~1e-7)."""
    n = 32768
    t, s = _clusters(n, 31, k=4, sigma=0.1), _clusters(n, 32, k=4, sigma=0.1)
    w = np.random.default_rng(33).uniform(-1, 1, n)
    ctx.set_kernel("inv_r_safe")
    mixed, used = ctx.solve(t, s, w, poly_ord=5, depth=2, precision=prec)
    assert used == 2
    rows = np.random.default_rng(34).choice(n, 2048, replace=False)
    ex = ctx.exact_rows(rows, t, s, w)
    assert rel_l2(mixed[rows], ex) <= 1e-6, rel_l2(mixed[rows], ex)


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3"])
def test_dense_leaves_mixed_within_2x_plain(ctx, prec):
    """3-D clustered 1/r (16 Gaussians, sigma 0.02, 6 nodes/dim) at Depth 5:
    the occupied leaves hold several hundred sources each, so the mixed near
    field sums long leaf lists.  Against the FP64 exact sum the mixed error
    stays within 2x the plain FMM's."""
    n = 200000
    t, s = _clusters(n, 41), _clusters(n, 42)
    w = np.random.default_rng(43).uniform(-1, 1, n)
    ctx.set_kernel("inv_r_safe")
    plain, _ = ctx.solve(t, s, w, poly_ord=5, depth=5, precision="fp64")
    mixed, _ = ctx.solve(t, s, w, poly_ord=5, depth=5, precision=prec)
    rows = np.random.default_rng(44).choice(n, 2048, replace=False)
    ex = ctx.exact_rows(rows, t, s, w)
    e_plain, e_mixed = rel_l2(plain[rows], ex), rel_l2(mixed[rows], ex)
    assert e_mixed <= 2.0 * e_plain, (e_mixed, e_plain)


@pytest.mark.parametrize("prec", ["bf16x3", "tf32x3"])
def test_two_sm_m2l_matches_one_sm(ctx, prec):
    """The 2-SM tensor-core M2L (clusters of two CTAs, 256-row tiles, the
    operator split between the SM pair) against the 1-SM kernel: 300,000
    uniform 3-D points at Depth 6 give 128 tiles of 256 rows at the leaf level,
    enough for every cluster, so that level takes the 2-SM kernel.  Each row's
    products are accumulated in the same order either way: the results agree
    to FP32 rounding (1e-6) and both stay within 1e-5 of the plain FP64 FMM."""
    r = np.random.default_rng(51)
    n = 300000
    t, s, w = r.random((n, 3)), r.random((n, 3)), r.uniform(-1, 1, n)
    ctx.set_kernel("inv_r_safe")
    try:
        ctx.set_m2l_options(pair=0)
        one, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision=prec)
        ctx.set_m2l_options(pair=1)
        two, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision=prec)
    finally:
        ctx.set_m2l_options()
    plain, _ = ctx.solve(t, s, w, poly_ord=5, depth=6, precision="fp64")
    print(f"{prec}: 2-SM vs 1-SM rel-L2 {rel_l2(two, one):.3e} (bit-identical: {np.array_equal(two, one)})")
    assert rel_l2(two, one) <= 1e-6, rel_l2(two, one)
    assert rel_l2(two, plain) <= 1e-5 and rel_l2(one, plain) <= 1e-5


@pytest.mark.parametrize("pair", [0, 1])
@pytest.mark.parametrize("d,po,depth,R", [(2, 4, 6, 16), (3, 5, 6, 1)])
def test_m2l_units_per_stage_bit_identical(ctx, pair, d, po, depth, R):
    """Pipeline stages of several (slot, K chunk) units (one barrier wait and
    one MMA commit per stage) issue the same MMAs into the same accumulators
    in the same order as stages of one unit: the results are bit-identical
    for 1 to 4 units per stage, in the 1-SM and the 2-SM kernel.  Covers the
    2-D multiquadric with 5 nodes (P = 25, one K chunk per slot, 16 rhs) and
    3-D 1/r with 6 nodes (P = 216, 7 K chunks per slot), where drain groups of
    14 units end in a partly filled stage for 3 and 4 units."""
    r = np.random.default_rng(61)
    n = 200000
    t, s = r.random((n, d)), r.random((n, d))
    W = r.standard_normal((R, n)) if R > 1 else r.uniform(-1, 1, n)
    if d == 2:
        ctx.set_kernel("multiquadric", 1e-4)
    else:
        ctx.set_kernel("inv_r_safe")
    out = {}
    try:
        for units in (1, 2, 3, 4):
            ctx.set_m2l_options(pair=pair, units=units)
            out[units], _ = ctx.solve(t, s, W, poly_ord=po, depth=depth, precision="bf16x3")
    finally:
        ctx.set_m2l_options()
    for units in (2, 3, 4):
        assert np.array_equal(out[units], out[1]), (units, rel_l2(out[units], out[1]))
