"""Host-side checks that need no GPU: the C-ABI library loads and exports
every declared symbol, the pyfmma drop-in validates like the reference
binding, and unsupported paths fail loudly."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fmma_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmma_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from fmma_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert set(syms) <= set(_lib.SIGNATURES), set(syms) - set(_lib.SIGNATURES)


def test_default_depth_matches_reference_formula(oracle):
    from fmma_b200 import _lib
    L = _lib.load()
    for nt, d in ((1, 1), (20, 2), (4096, 1), (10 ** 6, 2), (2 ** 22, 3), (12345, 3)):
        assert L.fmma_default_depth(nt, d) == oracle.default_depth(nt, d)


def test_stage_names():
    from fmma_b200 import _lib
    L = _lib.load()
    names = [L.fmma_stage_name(i).decode() for i in range(_lib.NUM_STAGES)]
    assert names == ["tree", "P2M", "M2M", "M2L", "L2L", "L2P", "P2P", "exact", "total"]


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import fmma_b200
    with pytest.raises(fmma_b200.FmmaError) as e:
        fmma_b200.Context(0)
    assert e.value.status == 6  # FMMA_ERR_NO_DEVICE


def test_pyfmma_shape_errors_like_reference_binding():
    import pyfmma
    f = pyfmma.fmmad2()
    t = np.zeros((5, 2))
    s = np.zeros((4, 2))
    ans = np.zeros(5)
    with pytest.raises(RuntimeError, match="target shape must be 2"):
        f.solve(np.zeros(5), s, ans)
    with pytest.raises(RuntimeError, match="target dimension must be 2"):
        f.solve(np.zeros((5, 3)), s, ans)
    with pytest.raises(RuntimeError, match="ans num 4 is different from target num 5"):
        f.solve(t, s, np.zeros(4))
    with pytest.raises(RuntimeError, match="source num 4 is different from source_weight num 3"):
        f.solve(t, np.zeros(3), s, ans)
    with pytest.raises(TypeError):
        f.solve(t, s, np.zeros(5, dtype=np.float32))


def test_pyfmma_rejects_python_callables_and_unknown_solvers():
    import pyfmma
    f = pyfmma.fmmad1()
    with pytest.raises(TypeError):
        f.set_fn2(lambda x, y: 1.0)
    with pytest.raises(TypeError):
        pyfmma.fmmad2().set_fn1(pyfmma.kernels.inv_diff)
    f.set_solver_type("bogus")
    with pytest.raises(RuntimeError, match="not undefined"):
        f.solve(np.zeros((3, 1)), np.zeros((3, 1)), np.zeros(3))
    assert f.check_blas() is False


def test_pyfmma_classes_exist():
    import pyfmma
    for name in ("fmmad1", "fmmaf1", "fmmad2", "fmmaf2", "fmmad3", "fmmaf3"):
        cls = getattr(pyfmma, name)
        for m in ("solve", "check_blas", "set_fn1", "set_fn2", "set_solver_type", "set_nrn_N", "set_poly_ord",
                  "set_Depth", "set_trans_sym_flag"):
            assert callable(getattr(cls, m))
