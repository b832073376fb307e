"""GPU tree build: binning bit-exact with the reference's P2M lists, and the
far/near interaction lists equal to the reference's (src/fmm_core.cpp:15-115)
restricted to boxes that hold sources."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d", [1, 2, 3])
def test_binning_bit_exact(ctx, oracle, d):
    g = golden(f"bins_d{d}")
    tb, sb, o, L = ctx.tree_export(g["tgt"], g["src"], int(g["depth"]))
    assert np.array_equal(o, g["origin"]) and L == float(g["Len"])
    assert np.array_equal(sb, g["src_box"])
    assert np.array_equal(tb, oracle.bin_points(d, int(g["depth"]), g["tgt"], o, L))


@pytest.mark.parametrize("d,depth", [(1, 9), (2, 6), (3, 5)])
def test_binning_on_box_faces(ctx, oracle, d, depth):
    # coordinates on exact multiples of the leaf width stress the division
    r = np.random.default_rng(d)
    N = 1 << (depth - 1)
    t = r.integers(0, N + 1, (5000, d)) / N
    s = r.integers(0, N + 1, (5000, d)) / N * 0.999 + 1e-3
    tb, sb, o, L = ctx.tree_export(t, s, depth)
    assert np.array_equal(tb, oracle.bin_points(d, depth, t, o, L))
    assert np.array_equal(sb, oracle.bin_points(d, depth, s, o, L))


@pytest.mark.parametrize("d,depth,clustered", [(1, 8, False), (2, 6, False), (3, 5, False), (3, 6, True)])
def test_interaction_lists(ctx, oracle, d, depth, clustered):
    r = np.random.default_rng(100 + d)
    n = 4000
    if clustered:
        c = r.uniform(0.2, 0.8, (3, d))
        t = np.clip(c[r.integers(0, 3, n)] + 0.04 * r.standard_normal((n, d)), 0, 1)
        s = np.clip(c[r.integers(0, 3, n)] + 0.04 * r.standard_normal((n, d)), 0, 1)
    else:
        t, s = r.random((n, d)), r.random((n, d))
    ctx.set_kernel("inv_r_safe" if d > 1 else "inv_diff")
    ctx.solve(t, s, None, poly_ord=1, depth=depth)
    o, L = oracle.origin_len(d, t, s)
    for level in range(2, depth):
        srcbox = set(oracle.bin_points(d, level + 1, s, o, L).tolist())
        tgtbox = sorted(set(oracle.bin_points(d, level + 1, t, o, L).tolist()))
        for box in r.choice(tgtbox, min(12, len(tgtbox)), replace=False):
            want = [b for b in oracle.far_list(d, int(box), 1 << level).tolist() if b in srcbox]
            got = ctx.interaction_list(level, int(box)).tolist()
            assert got == want, (level, box)
    leaf = depth - 1
    srcbox = set(oracle.bin_points(d, depth, s, o, L).tolist())
    tgtbox = sorted(set(oracle.bin_points(d, depth, t, o, L).tolist()))
    for box in r.choice(tgtbox, min(20, len(tgtbox)), replace=False):
        want = [b for b in oracle.near_list(d, int(box), 1 << leaf).tolist() if b in srcbox]
        assert ctx.near_list(int(box)).tolist() == want


def test_leaf_occupancy_and_depth_rule(ctx):
    import fmma_b200
    r = np.random.default_rng(12)
    t, s = r.random((20000, 2)), r.random((20000, 2))
    L = fmma_b200.choose_depth(ctx, t, s, 64)
    mt, ms = ctx.max_leaf_occupancy(t, s, L)
    assert mt <= 64 and ms <= 64
    mt2, ms2 = ctx.max_leaf_occupancy(t, s, L - 1)
    assert mt2 > 64 or ms2 > 64
