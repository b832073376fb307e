"""The oracle (C restatement) against the golden vectors made by the compiled
reference, against the compiled reference itself, and against the closed
forms of the reference's own math tests.  CPU only."""
import math

import numpy as np
import pytest

from conftest import golden, golden_names, rel_l2, rel_rms

FMM_CASES = [n for n in golden_names() if not n.startswith(("bins", "f", "tree", "nrnmm", "cheb"))]


@pytest.mark.parametrize("name", FMM_CASES)
def test_oracle_fmm_matches_golden(oracle, name):
    g = golden(name)
    d = int(g["dim"])
    out, used = oracle.fmm(d, int(g["kernel"]), float(g["p0"]), int(g["poly_ord"]), int(g["depth"]),
                           int(g["trans_sym"]), g["tgt"], g["src"], g.get("w"))
    assert used == int(g["depth_used"])
    # same loop order as the reference: agreement to the last bit is expected
    assert rel_l2(out, g["fmm"]) <= 1e-15
    assert np.array_equal(out, g["fmm"]) or np.max(np.abs(out - g["fmm"])) <= 1e-14 * np.max(np.abs(g["fmm"]))


@pytest.mark.parametrize("name", [n for n in FMM_CASES if "default" not in n and "L7" not in n])
def test_oracle_exact_matches_golden(oracle, name):
    g = golden(name)
    if "exact" not in g:
        pytest.skip("no exact vector")
    out = oracle.exact(int(g["dim"]), int(g["kernel"]), float(g["p0"]), g["tgt"], g["src"], g.get("w"))
    assert rel_l2(out, g["exact"]) <= 1e-15


@pytest.mark.parametrize("d", [1, 2, 3])
def test_oracle_binning_matches_golden(oracle, d):
    g = golden(f"bins_d{d}")
    o, L = oracle.origin_len(d, g["tgt"], g["src"])
    assert np.array_equal(o, g["origin"]) and L == float(g["Len"])
    box = oracle.bin_points(d, int(g["depth"]), g["src"], o, L)
    assert np.array_equal(box, g["src_box"])


@pytest.mark.parametrize("d,kid,po,depth,ts,n", [
    (1, 2, 7, 8, 0, 1500), (1, 0, 3, 6, 1, 700), (2, 3, 5, 5, 1, 2500), (2, 7, 3, 4, 0, 900),
    (3, 1, 3, 4, 1, 1500), (3, 5, 2, 4, 0, 800),
])
def test_oracle_bit_exact_vs_compiled_reference(oracle, ref, d, kid, po, depth, ts, n):
    r = np.random.default_rng(1000 + 7 * d + kid)
    t, s, w = r.random((n, d)), r.random((n, d)), r.uniform(-1, 1, n)
    p0 = 1e-4 if kid == 5 else 0.01
    a, _ = oracle.fmm(d, kid, p0, po, depth, ts, t, s, w)
    b, _ = ref.solve(d, "fmm", kid, p0, po, depth, ts, t, s, w)
    assert np.array_equal(a, b)


def test_chebyshev_closed_forms(oracle):
    # test/src/math/common.cpp:10-42
    for x in np.linspace(-1, 1, 41):
        assert abs(oracle.chebyshev(0, x) - 1.0) < 1e-12
        assert abs(oracle.chebyshev(1, x) - x) < 1e-12
        assert abs(oracle.chebyshev(2, x) - (2 * x * x - 1)) < 1e-12
        assert abs(oracle.chebyshev(3, x) - (4 * x ** 3 - 3 * x)) < 1e-12


def test_schebyshev_interpolation_converges(oracle):
    # test/src/math/kernel_approx.cpp: interpolating a smooth function on n nodes converges
    f = lambda x: 1.0 / (x + 3.0)
    errs = []
    for n in (2, 4, 8, 12):
        nodes = [math.cos((2 * k + 1) / (2 * n) * math.pi) for k in range(n)]
        xs = np.linspace(-1, 1, 101)
        approx = [sum(f(nodes[k]) * oracle.schebyshev(n, nodes[k], x) for k in range(n)) for x in xs]
        errs.append(max(abs(a - f(x)) for a, x in zip(approx, xs)))
    assert errs[-1] < 1e-6 and all(errs[i + 1] < errs[i] for i in range(len(errs) - 1))


def test_default_depth(oracle):
    for nt, d in ((1, 1), (2, 1), (20, 2), (4096, 1), (10 ** 6, 2), (2 ** 22, 3)):
        assert oracle.default_depth(nt, d) == max(1, int(math.log(nt) / d) + 1)


@pytest.mark.parametrize("d", [1, 2, 3])
def test_far_list_shape(oracle, d):
    N = 16
    nfar = 6 ** d - 3 ** d
    for box in np.random.default_rng(d).integers(0, N ** d, 40):
        lst = oracle.far_list(d, int(box), N)
        assert len(lst) <= nfar and len(set(lst.tolist())) == len(lst)
        c = np.array(np.unravel_index(int(box), (N,) * d))
        for b in lst:
            cb = np.array(np.unravel_index(int(b), (N,) * d))
            assert np.max(np.abs(cb - c)) >= 2 and np.all(np.abs(cb // 2 - c // 2) <= 1)
        assert list(lst) == sorted(lst)
        near = oracle.near_list(d, int(box), N)
        assert int(box) in near.tolist() and len(near) <= 3 ** d


@pytest.mark.parametrize("d,po,kid", [(1, 3, 0), (2, 3, 0), (2, 4, 6)])
def test_oracle_fmm_accuracy_like_reference_tests(oracle, d, po, kid):
    # test/src/fmma/fmm.cpp:10-61: rel-RMS vs exact below 1e-3 at Depth 3
    r = np.random.default_rng(5)
    t, s = r.random((20, d)) - 0.5, r.random((10, d)) - 0.5
    a, _ = oracle.fmm(d, kid, 0.0, po, 3, 1 if kid == 6 else 0, t, s)
    e = oracle.exact(d, kid, 0.0, t, s)
    assert rel_rms(a, e) < 1e-3


@pytest.mark.parametrize("name", ["tree_inv_diff_d1", "tree_log_r_d2", "tree_inv_r_safe_d3",
                                  "tree_gaussian_d2_default_depth"])
def test_oracle_tree_matches_reference_golden(oracle, name):
    """The C restatement of the tree solver (src/tree.cpp:12-100, M2P at
    src/fmm_core.cpp:624-661) against the compiled reference's outputs."""
    g = golden(name)
    d = int(g["dim"])
    w = g["w"] if "w" in g else None
    got, used = oracle.tree(d, int(g["kernel"]), float(g["p0"]), int(g["poly_ord"]), int(g["depth"]),
                            g["tgt"], g["src"], w)
    assert used == int(g["depth_used"])
    assert np.array_equal(got, g["tree"])


NRNMM_F64 = ["nrnmm_inv_r_d1", "nrnmm_sum_r2_d2", "nrnmm_sum2_r2_d2", "nrnmm_inv_diff_d1", "nrnmm_inv_r_safe_d3",
             "nrnmm_gaussian_d2_default_nrn", "nrnmm_clustered_d3"]


@pytest.mark.parametrize("name", NRNMM_F64)
def test_oracle_nrnmm_matches_reference_golden(oracle, name):
    """The C restatement of the nrnmm solver (src/nrnmm.cpp:13-102) against
    the compiled reference's outputs: identical to the last bit."""
    g = golden(name)
    d = int(g["dim"])
    w = g["w"] if "w" in g else None
    got, used = oracle.nrnmm(d, int(g["kernel"]), float(g["p0"]), int(g["poly_ord"]), int(g["nrn"]),
                             g["tgt"], g["src"], w)
    assert used == int(g["nrn_used"])
    assert np.array_equal(got, g["nrnmm"])


@pytest.mark.parametrize("d,kid,po,nrn", [(1, 0, 2, 3), (2, 0, 2, 3), (1, 6, 4, 6), (2, 7, 5, 6)])
def test_oracle_nrnmm_accuracy_like_reference_tests(oracle, d, kid, po, nrn):
    # test/src/fmma/nrnmm.cpp: rel-RMS vs exact below 1e-3
    r = np.random.default_rng(9)
    scale = 1.0 if kid == 0 else 5.0
    t, s = (r.random((20, d)) - 0.5) * scale, (r.random((10, d)) - 0.5) * scale
    w = None if kid == 0 else r.random(10)
    a, _ = oracle.nrnmm(d, kid, 0.0, po, nrn, t, s, w)
    e = oracle.exact(d, kid, 0.0, t, s, w)
    assert rel_rms(a, e) < 1e-3


def test_oracle_nrnmm_default_grid(oracle):
    # (int)(sqrt(3) * M^(1/(2 DIM))) + 1 with M the source count (src/nrnmm.cpp:20-22)
    for ns, d in [(1, 1), (300, 2), (10 ** 6, 3), (12345, 1)]:
        assert oracle.default_nrn(ns, d) == int(np.sqrt(3.0) * ns ** (1.0 / (2 * d))) + 1


CHEB_CASES = ["cheb_t2_d1", "cheb_t1t3_d2", "cheb_exp_cos_d1", "cheb_inv1p_d2", "cheb_inv1p_d3", "cheb_len2_d3",
              "cheb_exp_cos_d2"]


@pytest.mark.parametrize("name", CHEB_CASES)
def test_oracle_cheb_predict_matches_reference(oracle, name):
    """predict (src/chebyshev_approx.cpp:88-101) restated: identical to the
    compiled reference's predictions for the same coefficients."""
    g = golden(name)
    got = oracle.cheb_eval(int(g["dim"]), int(g["nth"]), g["coef"], g["pts"])
    assert np.array_equal(got, g["predict"])


@pytest.mark.parametrize("name", CHEB_CASES)
def test_oracle_cheb_fit_solves_reference_system(oracle, name):
    """The direct solve interpolates the node values to rounding; the
    reference's GCR coefficients lie within its stopping rule of it (squared
    residual 1e-6 on a system whose matrix has singular values >= 1)."""
    g = golden(name)
    dim, nth = int(g["dim"]), int(g["nth"])
    coef = oracle.cheb_fit(dim, nth, g["values"])
    n = nth + 1
    idx = np.arange(n ** dim)
    x = np.cos((2 * np.arange(n) + 1) / (2 * n) * np.pi)
    nodes = np.stack([x[(idx // n ** q) % n] for q in range(dim)], axis=1)
    fit = oracle.cheb_eval(dim, nth, coef, nodes)
    assert np.max(np.abs(fit - g["values"])) <= 1e-12 * max(1.0, np.max(np.abs(g["values"])))
    assert np.linalg.norm(coef - g["coef"]) <= 1e-3
