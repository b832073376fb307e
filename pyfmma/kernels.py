"""Built-in kernel handles for ``set_fn1`` / ``set_fn2``.

The reference binding accepts any Python callable (cpython/pyfmma.cpp:149-151)
and calls back into the interpreter for every kernel evaluation.  Kernels here
run on the GPU, so a Python callable cannot be used; pass one of these handles
instead.  Each handle names a device functor of libfmma_b200.
"""
from __future__ import annotations

from dataclasses import dataclass

from fmma_b200 import _lib


@dataclass(frozen=True)
class Kernel:
    """A built-in interaction kernel f(x, y) with its parameter."""
    kernel_id: int
    p0: float = 0.0
    name: str = ""
    translation_invariant: bool = True

    def __repr__(self) -> str:
        return f"pyfmma.kernels.{self.name}(p0={self.p0})" if self.p0 else f"pyfmma.kernels.{self.name}"


# 1/|x-y| without a guard: the reference default functor (include/fmma/fmma.hpp:55-63)
inv_r = Kernel(_lib.KERNEL_INV_R, 0.0, "inv_r")
# 1/|x-y|, 0 at coincidence
laplace = Kernel(_lib.KERNEL_INV_R_SAFE, 0.0, "laplace")
# 1/(x-y) in 1D, 0 at coincidence
inv_diff = Kernel(_lib.KERNEL_INV_DIFF, 0.0, "inv_diff")
# log|x-y|, 0 at coincidence
log_r = Kernel(_lib.KERNEL_LOG_R, 0.0, "log_r")
# sum_d (x-y)_d / |x-y|^2 (test/src/fmma/fmm.cpp:82-91)
sum_over_r2 = Kernel(_lib.KERNEL_SUM_OVER_R2, 0.0, "sum_over_r2")
# |x+y|^2 / |x-y|^2 (test/src/fmma/fmm.cpp:151-160), not translation invariant
sum2_over_r2 = Kernel(_lib.KERNEL_SUM2_OVER_R2, 0.0, "sum2_over_r2", translation_invariant=False)


def gaussian(p0: float = 0.01) -> Kernel:
    """exp(-|x-y|^2 / p0)."""
    return Kernel(_lib.KERNEL_GAUSSIAN, float(p0), "gaussian")


def multiquadric(p0: float = 1e-4) -> Kernel:
    """sqrt(|x-y|^2 + p0)."""
    return Kernel(_lib.KERNEL_MULTIQUADRIC, float(p0), "multiquadric")
