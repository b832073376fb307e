import glob
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import ORACLE_SO, Oracle
    if not os.path.exists(ORACLE_SO):
        # oracle only: the reference tree is not read here
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=/nonexistent",
                               "_build/liboracle.so"])
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("compiled reference (oracle/_ref) not built")
    return Reference()


@pytest.fixture(scope="session")
def ctx():
    import fmma_b200
    return fmma_b200.default_context(0)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names(prefix=""):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def rel_rms(a, e):
    """The reference's per-point relative RMS (test/src/fmma/fmm.cpp:46-51)."""
    a = np.asarray(a, dtype=np.float64)
    e = np.asarray(e, dtype=np.float64)
    return float(np.sqrt(np.mean(((a - e) / e) ** 2)))
