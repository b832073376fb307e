"""pyfmma — drop-in for the reference's pybind11 module (cpython/pyfmma.cpp),
running the exact, fmm, tree and nrnmm solvers on a B200 through libfmma_b200.

Classes ``fmmad1, fmmaf1, fmmad2, fmmaf2, fmmad3, fmmaf3`` keep the reference's
methods (cpython/pyfmma.cpp:145-156): ``solve`` (with and without weights),
``check_blas``, ``set_fn1``, ``set_fn2``, ``set_solver_type``, ``set_nrn_N``,
``set_poly_ord``, ``set_Depth``, ``set_trans_sym_flag``.  Differences:

* ``set_fn1`` / ``set_fn2`` take a handle from :mod:`pyfmma.kernels` or a C++
  expression string (compiled for the device at run time); a Python callable
  raises TypeError (it cannot run on the device).
* solver types "tree" (built-in kernels) and "nrnmm" run on the GPU in FP64;
  "exact_matvec" runs the exact solver (same sum, src/fmma.cpp:103-141).
* an ``ans`` array of the wrong dtype raises TypeError instead of being left
  unwritten.
* extensions: ``set_precision``, multi-RHS weights of shape (R, M) with ``ans``
  of shape (R, N), CUDA torch tensors (zero copy), ``stage_times``.

The GIL is released during ``solve`` (ctypes foreign calls release it).
"""
from __future__ import annotations

import numpy as np

import fmma_b200
from fmma_b200 import FmmaError

from . import kernels
from .kernels import Kernel

__version__ = "0.1.2"

_SOLVER_ALIASES = {"exact": "exact", "exact_matvec": "exact", "fmm": "fmm", "tree": "tree", "nrnmm": "nrnmm"}


class _FMMA:
    TYPE = np.float64
    DIM = 1

    def __init__(self):
        self._solver = "exact"          # include/fmma/fmma.hpp:90
        self._nrn_N = -1                # :98
        self._poly_ord = 1              # :106
        self._Depth = -1                # :114
        self._trans_sym_flag = 0        # :122
        self._kernel = kernels.inv_r    # :55-63
        self._precision = "fp64"
        self.time_log = {}
        self._device = 0

    # -- setters (include/fmma/fmma.hpp:65-127) --------------------------------
    def set_fn1(self, fn):
        """f(x - y): a pyfmma.kernels handle, or a C++ expression string in
        dx[q] = x[q] - y[q], r2 = |x - y|^2 and r (compiled for the device)."""
        self._set_fn(fn, translation_invariant=True)

    def set_fn2(self, fn):
        """f(x, y): a pyfmma.kernels handle, or a C++ expression string in
        x[q], y[q] (and dx[q], r2, r), compiled for the device."""
        self._set_fn(fn, translation_invariant=False)

    def _set_fn(self, fn, translation_invariant):
        if isinstance(fn, str):
            # an expression kernel lives on a context of this object, compiled once here
            ctx = fmma_b200.Context(self._device)
            try:
                ctx.set_kernel_expr(fn, translation_invariant)
            except FmmaError as e:
                ctx.close()
                raise RuntimeError(str(e)) from e
            self._drop_own_context()
            self._own_ctx = ctx
            self._kernel = fn
            return
        if not isinstance(fn, Kernel):
            raise TypeError(
                "set_fn1/set_fn2 take a kernel handle from pyfmma.kernels (e.g. pyfmma.kernels.laplace) or a "
                "C++ expression string such as 'exp(-r2 / 0.01)'; Python callables cannot run on the GPU")
        if fn.kernel_id == kernels.inv_diff.kernel_id and self.DIM != 1:
            raise TypeError("inv_diff is a one-dimensional kernel")
        self._drop_own_context()
        self._kernel = fn

    def _drop_own_context(self):
        ctx = getattr(self, "_own_ctx", None)
        if ctx is not None:
            ctx.close()
        self._own_ctx = None

    def set_solver_type(self, new_type: str):
        self._solver = str(new_type)

    def set_nrn_N(self, n: int):
        self._nrn_N = int(n)

    def set_poly_ord(self, p: int):
        self._poly_ord = int(p)

    def set_Depth(self, d: int):
        self._Depth = int(d)

    def set_trans_sym_flag(self, f: int):
        self._trans_sym_flag = int(f)

    def set_precision(self, p: str):
        if p not in fmma_b200.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(fmma_b200.PRECISIONS)}")
        self._precision = p

    def set_device(self, device: int):
        self._device = int(device)

    def check_blas(self) -> bool:
        return False

    # -- solve (cpython/pyfmma.cpp:16-135) ------------------------------------
    def solve(self, target, *args):
        if len(args) == 3:
            source_weight, source, ans = args
        elif len(args) == 2:
            source, ans = args
            source_weight = None
        else:
            raise TypeError("solve(target, [source_weight,] source, ans)")
        self._check_shapes(target, source_weight, source, ans)
        solver = _SOLVER_ALIASES.get(self._solver)
        if solver is None:
            raise RuntimeError(f"ERROR : solve type {self._solver} not undefined")
        own = getattr(self, "_own_ctx", None)
        ctx = own if own is not None else fmma_b200.default_context(self._device)
        with ctx.lock:
            if own is None:
                ctx.set_kernel(self._kernel.kernel_id, self._kernel.p0)
            # nrnmm takes nrn_N in the depth slot (src/nrnmm.cpp:20-22)
            depth = self._nrn_N if solver == "nrnmm" else self._Depth
            try:
                _, used = ctx.solve(target, source, source_weight, solver=solver, poly_ord=self._poly_ord,
                                    depth=depth, trans_sym=self._trans_sym_flag,
                                    precision=self._precision, out=ans)
            except FmmaError as e:
                raise RuntimeError(str(e)) from e
            if solver in ("fmm", "tree") and self._Depth <= 0 and target.shape[0] > 0:
                self._Depth = used    # sticky default Depth (src/fmm.cpp:23-28)
            if solver == "nrnmm" and self._nrn_N <= 0:
                self._nrn_N = used    # sticky default nrn_N
            st = ctx.stage_times()
        self.time_log[f"total time({self._solver})"] = st["total"]
        for k in ("P2M", "M2M", "M2L", "L2L", "L2P", "P2P"):
            if st[k]:
                self.time_log[k] = self.time_log.get(k, 0.0) + st[k]

    def stage_times(self) -> dict:
        return fmma_b200.default_context(self._device).stage_times()

    def _check_shapes(self, target, source_weight, source, ans):
        def nd(x):
            return len(x.shape)
        if nd(target) != 2:
            raise RuntimeError(f"target shape must be 2 but {nd(target)}")
        if source_weight is not None and nd(source_weight) not in (1, 2):
            raise RuntimeError(f"source_weight shape must be 2 but {nd(source_weight)}")
        if nd(source) != 2:
            raise RuntimeError(f"source shape must be 2 but {nd(source)}")
        want_ans = 1 if (source_weight is None or nd(source_weight) == 1) else 2
        if nd(ans) != want_ans:
            raise RuntimeError(f"ans shape must be {want_ans} but {nd(ans)}")
        if target.shape[1] != self.DIM:
            raise RuntimeError(f"target dimension must be {self.DIM} but {target.shape[1]}")
        if source.shape[1] != self.DIM:
            raise RuntimeError(f"source dimension must be {self.DIM} but {source.shape[1]}")
        if ans.shape[-1] != target.shape[0]:
            raise RuntimeError(f"ans num {ans.shape[-1]} is different from target num {target.shape[0]}")
        if source_weight is not None and source.shape[0] != source_weight.shape[-1]:
            raise RuntimeError(f"source num {source.shape[0]} is different from source_weight num "
                               f"{source_weight.shape[-1]}")
        for name, x in (("target", target), ("source", source), ("ans", ans), ("source_weight", source_weight)):
            if x is None:
                continue
            dt = getattr(x, "dtype", None)
            ok = (dt == self.TYPE) if isinstance(x, np.ndarray) else (str(dt) == f"torch.{np.dtype(self.TYPE).name}")
            if not ok:
                raise TypeError(f"{name} must have dtype {np.dtype(self.TYPE).name}")


def _make(type_char, dim):
    t = np.float64 if type_char == "d" else np.float32
    return type(f"fmma{type_char}{dim}", (_FMMA,), {"TYPE": t, "DIM": dim,
                                                     "__doc__": f"FMMA<{np.dtype(t).name},{dim}> on the GPU."})


fmmad1 = _make("d", 1)
fmmaf1 = _make("f", 1)
fmmad2 = _make("d", 2)
fmmaf2 = _make("f", 2)
fmmad3 = _make("d", 3)
fmmaf3 = _make("f", 3)

__all__ = ["fmmad1", "fmmaf1", "fmmad2", "fmmaf2", "fmmad3", "fmmaf3", "kernels", "Kernel"]
