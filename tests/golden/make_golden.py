"""Generates the golden vectors in tests/golden/*.npz from the reference
library compiled from its own sources (oracle/_ref/libfmma_ref.so, built by
`make -C oracle`).  Run from the repository root:

    python tests/golden/make_golden.py

Each file stores the inputs (seeded), the parameters and the reference's own
outputs of FMMA<T,DIM>::solve for solver "fmm" and "exact" (tree_*: "tree",
nrnmm_*: "nrnmm", the latter after the reference's test/src/fmma/nrnmm.cpp;
cheb_*: CHEBYSHEV_APPROX fits and predictions).  The cases follow
the reference's tests (test/src/fmma/fmm.cpp, common.cpp: kernels, orders,
depths) and the 1-D configuration of the benchmark (4096 points, 8 nodes).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
K = dict(inv_r=0, inv_r_safe=1, inv_diff=2, log_r=3, gaussian=4, multiquadric=5, sum_over_r2=6, sum2_over_r2=7)


def case(name, d, kernel, p0, poly_ord, depth, trans_sym, tgt, src, w, dtype=np.float64, exact=True):
    ref = Reference()
    kid = K[kernel]
    fmm, used = ref.solve(d, "fmm", kid, p0, poly_ord, depth, trans_sym, tgt, src, w, dtype=dtype)
    out = dict(dim=d, kernel=kid, p0=p0, poly_ord=poly_ord, depth=depth, depth_used=used, trans_sym=trans_sym,
               tgt=np.asarray(tgt, dtype=dtype), src=np.asarray(src, dtype=dtype), fmm=fmm)
    if w is not None:
        out["w"] = np.asarray(w, dtype=dtype)
    if exact:
        ex, _ = ref.solve(d, "exact", kid, p0, poly_ord, depth, trans_sym, tgt, src, w, dtype=dtype)
        out["exact"] = ex
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(name, d, kernel, "depth", used, "n", len(tgt))


def tree_case(name, d, kernel, p0, poly_ord, depth, tgt, src, w, dtype=np.float64):
    """The reference's tree solver (src/tree.cpp:12-100) on seeded inputs."""
    ref = Reference()
    kid = K[kernel]
    tree, used = ref.solve(d, "tree", kid, p0, poly_ord, depth, 0, tgt, src, w, dtype=dtype)
    out = dict(dim=d, kernel=kid, p0=p0, poly_ord=poly_ord, depth=depth, depth_used=used,
               tgt=np.asarray(tgt, dtype=dtype), src=np.asarray(src, dtype=dtype), tree=tree)
    if w is not None:
        out["w"] = np.asarray(w, dtype=dtype)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(name, d, kernel, "tree depth", used, "n", len(tgt))


def nrnmm_case(name, d, kernel, p0, poly_ord, nrn, tgt, src, w, dtype=np.float64):
    """The reference's nrnmm solver (src/nrnmm.cpp:13-102) on seeded inputs."""
    ref = Reference()
    kid = K[kernel]
    ans, used = ref.solve(d, "nrnmm", kid, p0, poly_ord, nrn, 0, tgt, src, w, dtype=dtype)
    out = dict(dim=d, kernel=kid, p0=p0, poly_ord=poly_ord, nrn=nrn, nrn_used=used,
               tgt=np.asarray(tgt, dtype=dtype), src=np.asarray(src, dtype=dtype), nrnmm=ans)
    if w is not None:
        out["w"] = np.asarray(w, dtype=dtype)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(name, d, kernel, "nrn", used, "n", len(tgt))


def main_nrnmm():
    r = np.random.default_rng(43)
    # test/src/fmma/nrnmm.cpp:10-61 (default 1/r, unweighted, poly_ord 2, nrn_N 3), more points
    nrnmm_case("nrnmm_inv_r_d1", 1, "inv_r", 0.0, 2, 3, r.random((400, 1)) - 0.5, r.random((300, 1)) - 0.5, None)
    nrnmm_case("nrnmm_inv_r_d2_f32", 2, "inv_r", 0.0, 2, 3, r.random((400, 2)) - 0.5, r.random((300, 2)) - 0.5,
               None, dtype=np.float32)
    # test/src/fmma/nrnmm.cpp:63-129 and :131-197 (poly_ord 4 / 5, nrn_N 6, points in [-2.5, 2.5))
    nrnmm_case("nrnmm_sum_r2_d2", 2, "sum_over_r2", 0.0, 4, 6, (r.random((1500, 2)) - 0.5) * 5,
               (r.random((1500, 2)) - 0.5) * 5, r.random(1500))
    nrnmm_case("nrnmm_sum2_r2_d2", 2, "sum2_over_r2", 0.0, 5, 6, (r.random((1500, 2)) - 0.5) * 5,
               (r.random((1500, 2)) - 0.5) * 5, r.random(1500))
    nrnmm_case("nrnmm_inv_diff_d1", 1, "inv_diff", 0.0, 7, 11, r.random((2000, 1)), r.random((2000, 1)),
               r.uniform(-1, 1, 2000))
    nrnmm_case("nrnmm_inv_r_safe_d3", 3, "inv_r_safe", 0.0, 3, 7, r.random((3000, 3)), r.random((3000, 3)),
               r.uniform(-1, 1, 3000))
    nrnmm_case("nrnmm_gaussian_d2_default_nrn", 2, "gaussian", 0.01, 4, -1, r.random((2000, 2)),
               r.random((2500, 2)), r.standard_normal(2500))
    nrnmm_case("nrnmm_log_r_d2_f32", 2, "log_r", 0.0, 4, 5, r.random((1500, 2)), r.random((1500, 2)),
               r.standard_normal(1500), dtype=np.float32)
    # clustered sources: most boxes of a 9^3 grid hold none
    c = r.random((6, 3))
    src = (c[r.integers(0, 6, 2500)] + 0.03 * r.standard_normal((2500, 3)))
    nrnmm_case("nrnmm_clustered_d3", 3, "multiquadric", 1e-3, 3, 9, r.random((2000, 3)), src,
               r.standard_normal(2500))


def main_cheb():
    """CHEBYSHEV_APPROX<double, dim> (src/chebyshev_approx.cpp:36-101): the
    reference's node values and coefficients for the shim's test functions
    (0 |x|^2, 1 1/(1+|x|^2), 2 exp(x0) cos(2 x_{d-1}), 3 T_a(x0) T_b(x1)),
    and its predictions at seeded points in [-1, 1]^dim."""
    ref = Reference()
    r = np.random.default_rng(47)
    for name, dim, nth, fid, a, b in [("cheb_t2_d1", 1, 10, 3, 2, 0), ("cheb_t1t3_d2", 2, 5, 3, 1, 3),
                                      ("cheb_exp_cos_d1", 1, 12, 2, 0, 0), ("cheb_inv1p_d2", 2, 8, 1, 0, 0),
                                      ("cheb_inv1p_d3", 3, 6, 1, 0, 0), ("cheb_len2_d3", 3, 5, 0, 0, 0),
                                      ("cheb_exp_cos_d2", 2, 14, 2, 0, 0)]:
        values, coef = ref.cheb_fit(dim, nth, fid, a, b)
        pts = r.uniform(-1.0, 1.0, (2000, dim))
        pred = ref.cheb_predict(dim, nth, coef, pts)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), dim=dim, nth=nth, fid=fid, a=a, b=b, values=values,
                            coef=coef, pts=pts, predict=pred)
        print(name, dim, nth, fid)


def main_tree():
    r = np.random.default_rng(41)
    tree_case("tree_inv_diff_d1", 1, "inv_diff", 0.0, 7, 6, r.random((1500, 1)), r.random((1500, 1)),
              r.uniform(-1, 1, 1500))
    tree_case("tree_log_r_d2", 2, "log_r", 0.0, 5, 5, r.random((2000, 2)), r.random((2000, 2)),
              r.standard_normal(2000))
    tree_case("tree_inv_r_safe_d3", 3, "inv_r_safe", 0.0, 3, 4, r.random((1500, 3)), r.random((1500, 3)),
              r.uniform(-1, 1, 1500))
    tree_case("tree_gaussian_d2_default_depth", 2, "gaussian", 0.01, 4, -1, r.random((1200, 2)),
              r.random((1200, 2)), None)
    tree_case("tree_multiquadric_d2_f32", 2, "multiquadric", 1e-4, 4, 5, r.random((1500, 2)), r.random((1500, 2)),
              r.standard_normal(1500), dtype=np.float32)


def main():
    # C1: 1-D, 4096 + 4096 points, separate seeds, 1/(x-y), 8 nodes, leaves <= 64 -> Depth 8
    t = np.random.default_rng(1).random((4096, 1))
    s = np.random.default_rng(2).random((4096, 1))
    w = np.random.default_rng(3).uniform(-1, 1, 4096)
    case("c1_inv_diff_L8", 1, "inv_diff", 0.0, 7, 8, 0, t, s, w)
    case("c1_inv_diff_L7_sym", 1, "inv_diff", 0.0, 7, 7, 1, t, s, w, exact=False)
    case("c1_inv_diff_default_depth", 1, "inv_diff", 0.0, 7, -1, 0, t, s, w, exact=False)

    # the reference's own test cases (test/src/fmma/fmm.cpp), seeded here
    for d in (1, 2):
        r = np.random.default_rng(10 + d)
        case(f"reftest_fmm_inv_r_d{d}", d, "inv_r", 0.0, 3, 3, 0,
             r.random((20, d)) - 0.5, r.random((10, d)) - 0.5, None)
        case(f"reftest_fmm_1_r2_d{d}", d, "sum_over_r2", 0.0, 4, 3, 1,
             (r.random((20, d)) - 0.5) * 5, (r.random((10, d)) - 0.5) * 5, r.random(10))
        case(f"reftest_fmm_sum2_r2_d{d}", d, "sum2_over_r2", 0.0, 5, 3, 0,
             (r.random((20, d)) - 0.5) * 5, (r.random((10, d)) - 0.5) * 5, r.random(10))

    # 2-D log r, 6 nodes, far field on levels 2..5
    r = np.random.default_rng(20)
    t, s = r.random((6000, 2)), r.random((6000, 2))
    case("d2_log_r_n6_L6", 2, "log_r", 0.0, 5, 6, 0, t, s, r.standard_normal(6000))
    case("d2_mq_n5_L5_sym", 2, "multiquadric", 1e-4, 4, 5, 1, t[:3000], s[:3000], r.standard_normal(3000))
    # non-translation-invariant kernel, per-pair M2L, levels 2..4
    case("d2_sum2_r2_n4_L5", 2, "sum2_over_r2", 0.0, 3, 5, 0, t[:2000] * 5 - 2.5, s[:2000] * 5 - 2.5,
         r.random(2000))

    # 3-D
    r = np.random.default_rng(30)
    t, s = r.random((3000, 3)), r.random((3000, 3))
    case("d3_inv_r_safe_n4_L4_sym", 3, "inv_r_safe", 0.0, 3, 4, 1, t, s, r.uniform(-1, 1, 3000))
    case("d3_gauss_n4_L4", 3, "gaussian", 0.01, 3, 4, 1, t[:2000], s[:2000], r.standard_normal(2000))
    # clustered 3-D (mixture of Gaussians clipped to the unit cube)
    r = np.random.default_rng(31)
    cen = r.uniform(0.1, 0.9, (4, 3))

    def blob(rr, n):
        k = rr.integers(0, 4, n)
        return np.clip(cen[k] + 0.05 * rr.standard_normal((n, 3)), 0.0, 1.0)

    case("d3_clustered_n3_L5", 3, "inv_r_safe", 0.0, 2, 5, 1, blob(np.random.default_rng(32), 3000),
         blob(np.random.default_rng(33), 3000), np.random.default_rng(34).uniform(-1, 1, 3000))

    # float instantiation: binning in float
    r = np.random.default_rng(40)
    case("f2_log_r_n5_L5", 2, "log_r", 0.0, 4, 5, 0, r.random((3000, 2)).astype(np.float32),
         r.random((3000, 2)).astype(np.float32), r.standard_normal(3000).astype(np.float32), dtype=np.float32)

    # binning fixture: source boxes as the reference's P2M lists them
    ref = Reference()
    r = np.random.default_rng(50)
    for d, depth in ((1, 9), (2, 7), (3, 6)):
        t = r.random((4000, d)) * 3 - 1
        s = r.random((4000, d)) * 3 - 1
        # points on box faces: multiples of the leaf width from the cube origin
        s[:500] = np.round(s[:500] * 64) / 64
        box, ol, _ = ref.p2m_bins(d, depth, 1, t, s, np.ones(len(s)))
        np.savez_compressed(os.path.join(OUT, f"bins_d{d}.npz"), dim=d, depth=depth, tgt=t, src=s, src_box=box,
                            origin=ol[:d], Len=ol[d])
        print("bins", d, depth)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "tree":
        main_tree()
    elif len(sys.argv) > 1 and sys.argv[1] == "nrnmm":
        main_nrnmm()
    elif len(sys.argv) > 1 and sys.argv[1] == "cheb":
        main_cheb()
    else:
        main()
        main_tree()
        main_nrnmm()
        main_cheb()
