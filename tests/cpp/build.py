"""Compiles tests/cpp/test_fmma_api.cu against the in-tree library."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(HERE, "test_fmma_api")


def build() -> str:
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from fmma_b200.build import nvcc
    src = os.path.join(HERE, "test_fmma_api.cu")
    hdrs = [os.path.join(ROOT, "include", "fmma", n) for n in ("fmma.hpp", "device.cuh")]
    lib = os.path.join(ROOT, "fmma_b200", "libfmma_b200.so")
    if os.path.exists(BIN) and os.path.getmtime(BIN) >= max(os.path.getmtime(p) for p in [src, lib, *hdrs]):
        return BIN
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "--expt-relaxed-constexpr",
           "--extended-lambda", "-I", os.path.join(ROOT, "include"), src, "-L", os.path.join(ROOT, "fmma_b200"),
           "-lfmma_b200", "-Xlinker", "-rpath,$ORIGIN/../../fmma_b200", "-o", BIN]
    subprocess.check_call(cmd)
    return BIN


if __name__ == "__main__":
    print(build())
