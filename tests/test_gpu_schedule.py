"""Schedule options: the choices the plan autotuner makes, set by hand on a
context (fmma_set_schedule_options).  Every leaf evaluation layout matches
the oracle on dense and sparse leaves with one and several rhs, including the
layouts the default rule would not pick for that density; every slot split of
the small tensor-core M2L levels agrees with the default split.

Tolerances: plain FP64 fmm vs the oracle, relative L2 <= 1e-12 (as the parity
tests); a split mode vs the default split, relative L2 <= 2e-6 (the FP32
partial sums of a tile regroup, as for a problem solved alone or inside a
forest) and vs plain FP64 <= 1e-5."""
import numpy as np
import pytest

import fmma_b200
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture()
def own_ctx():
    c = fmma_b200.Context(0)
    yield c
    c.close()


# (d, kernel id, poly_ord, Depth, points, rhs): targets per leaf
LEAF_CASES = [
    (3, 1, 5, 5, 20000, 1),  # ~5: sparse, one rhs (mode 2 runs the fused leaf L2L)
    (3, 4, 3, 3, 8000, 1),   # ~125: dense, one rhs
    (2, 3, 4, 4, 6000, 3),   # ~94: dense, three rhs
    (2, 3, 5, 7, 30000, 2),  # ~7: sparse, two rhs
]


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("d,kid,po,depth,n,R", LEAF_CASES)
def test_leaf_layouts_match_oracle(own_ctx, oracle, mode, d, kid, po, depth, n, R):
    r = np.random.default_rng(300 + 10 * d + kid)
    t, s = r.random((n, d)), r.random((n, d))
    W = r.uniform(-1, 1, (R, n))
    own_ctx.set_kernel(kid, 0.01)
    own_ctx.set_schedule_options(l2p_mode=mode)
    out, _ = own_ctx.solve(t, s, W if R > 1 else W[0], poly_ord=po, depth=depth)
    out = out.reshape(R, n)
    for k in range(R):
        ref, _ = oracle.fmm(d, kid, 0.01, po, depth, 0, t, s, np.ascontiguousarray(W[k]))
        assert rel_l2(out[k], ref) <= 1e-12, (k, rel_l2(out[k], ref))


@pytest.mark.parametrize("split", [1, 2, 3])
def test_m2l_split_modes_agree(own_ctx, split):
    r = np.random.default_rng(41)
    n = 40000
    t, s, w = r.random((n, 3)), r.random((n, 3)), r.uniform(-1, 1, n)
    own_ctx.set_kernel("inv_r_safe")
    plain, _ = own_ctx.solve(t, s, w, poly_ord=4, depth=5)
    base, _ = own_ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
    own_ctx.set_schedule_options(m2l_split=split)
    got, _ = own_ctx.solve(t, s, w, poly_ord=4, depth=5, precision="bf16x3")
    assert rel_l2(got, base) <= 2e-6, rel_l2(got, base)
    assert rel_l2(got, plain) <= 1e-5


def test_schedule_options_rejected_out_of_range(own_ctx):
    with pytest.raises(RuntimeError):
        own_ctx.set_schedule_options(m2l_split=4)
    with pytest.raises(RuntimeError):
        own_ctx.set_schedule_options(l2p_mode=-1)
