"""pyfmma drop-in on the GPU: the reference's Python usage against the
reference's own outputs."""
import numpy as np
import pytest

from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


def test_pyfmma_fmm_matches_reference_golden():
    import pyfmma
    g = golden("d2_log_r_n6_L6")
    f = pyfmma.fmmad2()
    f.set_fn2(pyfmma.kernels.log_r)
    f.set_solver_type("fmm")
    f.set_poly_ord(int(g["poly_ord"]))
    f.set_Depth(int(g["depth"]))
    ans = np.zeros(len(g["tgt"]))
    f.solve(g["tgt"], g["w"], g["src"], ans)
    assert rel_l2(ans, g["fmm"]) <= 1e-12
    assert f.time_log["total time(fmm)"] > 0


def test_pyfmma_sticky_default_depth():
    import pyfmma
    g = golden("c1_inv_diff_default_depth")
    f = pyfmma.fmmad1()
    f.set_fn1(pyfmma.kernels.inv_diff)
    f.set_solver_type("fmm")
    f.set_poly_ord(7)
    ans = np.zeros(len(g["tgt"]))
    f.solve(g["tgt"], g["w"], g["src"], ans)
    assert f._Depth == int(g["depth_used"])
    assert rel_l2(ans, g["fmm"]) <= 1e-12


def test_pyfmma_exact_default_solver_and_float():
    import pyfmma
    g = golden("f2_log_r_n5_L5")
    f = pyfmma.fmmaf2()
    f.set_fn2(pyfmma.kernels.log_r)
    ans = np.zeros(len(g["tgt"]), dtype=np.float32)
    f.solve(g["tgt"], g["w"], g["src"], ans)   # solver "exact" is the default
    assert rel_l2(ans, g["exact"]) <= 2e-6


def test_pyfmma_unweighted_3d_default_kernel():
    import pyfmma
    r = np.random.default_rng(0)
    t, s = r.random((500, 3)) - 0.5, r.random((400, 3)) - 0.5
    f = pyfmma.fmmad3()
    f.set_solver_type("fmm")
    f.set_poly_ord(3)
    f.set_Depth(3)
    a = np.zeros(500)
    f.solve(t, s, a)
    e = np.array([np.sum(1.0 / np.linalg.norm(s - x, axis=1)) for x in t])
    assert np.sqrt(np.mean(((a - e) / e) ** 2)) < 1e-3
