"""The C++ drop-in header (include/fmma/fmma.hpp, include/fmma/device.cuh)
on the GPU: the reference's own test programs ported to the header, user
__device__ functors and lambdas, error behaviour.  Runs the compiled program
tests/cpp/test_fmma_api (built by __graft_entry__.build or here with nvcc)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_cpp_api_program():
    sys.path.insert(0, os.path.join(HERE, "cpp"))
    from build import build
    exe = build()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    print(r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout
    assert r.stdout.count("PASS") >= 20
