"""fmma_b200 — B200 (sm_100a) implementation of FMMA's exact and fmm solvers.

Python side of the C ABI in include/fmma_b200.h.  Arrays may be numpy arrays
(host memory: the library stages them through the device) or CUDA torch
tensors (device memory, zero copy).  There is no CPU fallback: every solve runs
the CUDA kernels of libfmma_b200.so.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib
from ._lib import FmmaError, check

__all__ = ["Context", "FmmaError", "KERNELS", "PRECISIONS", "Plan", "SOLVERS", "cheb_nodes", "cheb_points", "choose_depth",
           "default_context"]

KERNELS = {
    "inv_r": _lib.KERNEL_INV_R,
    "inv_r_safe": _lib.KERNEL_INV_R_SAFE,
    "inv_diff": _lib.KERNEL_INV_DIFF,
    "log_r": _lib.KERNEL_LOG_R,
    "gaussian": _lib.KERNEL_GAUSSIAN,
    "multiquadric": _lib.KERNEL_MULTIQUADRIC,
    "sum_over_r2": _lib.KERNEL_SUM_OVER_R2,
    "sum2_over_r2": _lib.KERNEL_SUM2_OVER_R2,
}
PRECISIONS = {"fp64": _lib.PREC_FP64, "plain": _lib.PREC_FP64,
              "mixed": _lib.PREC_MIXED_TF32X3, "tf32x3": _lib.PREC_MIXED_TF32X3,
              "bf16x3": _lib.PREC_MIXED_BF16X3}
SOLVERS = {"exact": _lib.SOLVER_EXACT, "fmm": _lib.SOLVER_FMM, "tree": _lib.SOLVER_TREE,
           "nrnmm": _lib.SOLVER_NRNMM}


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class _Arr:
    """A pointer view of a numpy array or torch tensor."""

    def __init__(self, x, dtype, name):
        self.obj = x
        if x is None:
            self.ptr, self.kind, self.shape = None, None, None
            return
        if _is_torch(x):
            import torch
            want = torch.float64 if dtype == np.float64 else torch.float32
            if x.dtype != want:
                raise TypeError(f"{name}: expected {want}, got {x.dtype}")
            if not x.is_contiguous():
                raise ValueError(f"{name}: tensor must be contiguous")
            if x.is_cuda:
                self.ptr, self.kind = x.data_ptr(), _lib.MEM_DEVICE
            else:
                self.ptr, self.kind = x.data_ptr(), _lib.MEM_HOST
            self.shape = tuple(x.shape)
            return
        if not isinstance(x, np.ndarray):
            raise TypeError(f"{name}: expected a numpy array or torch tensor")
        if x.dtype != dtype:
            raise TypeError(f"{name}: expected dtype {np.dtype(dtype)}, got {x.dtype}")
        if not x.flags.c_contiguous:
            raise ValueError(f"{name}: array must be C-contiguous")
        self.ptr, self.kind, self.shape = x.ctypes.data, _lib.MEM_HOST, x.shape


def _mem_kind(*arrs) -> int:
    kinds = {a.kind for a in arrs if a.kind is not None}
    if len(kinds) > 1:
        raise ValueError("all arrays must live in the same memory (all host or all CUDA)")
    return kinds.pop() if kinds else _lib.MEM_HOST


class Context:
    """An fmma_ctx: one CUDA stream, device scratch and an operator cache.

    Not thread-safe (the same contract as the reference's FMMA object)."""

    def __init__(self, device: int = 0):
        self._L = _lib.load()
        h = C.c_void_p()
        check(self._L.fmma_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device
        self.lock = threading.RLock()
        self.kernel = ("inv_r", 0.0)
        self._xstream = None

    def set_allocator(self, alloc=None, free=None):
        """Routes the context's device scratch and operator cache through
        alloc(bytes, stream) -> device pointer (int; 0 when it cannot serve
        the request: the call then fails with FmmaError status 3, OOM) and
        free(ptr, bytes, stream).  No arguments: back to cudaMalloc/cudaFree.
        Switching releases the current scratch through the old allocator."""
        if alloc is None:
            with self.lock:
                check(self._L.fmma_set_allocator(self._h, None, None, None))
            self._alloc_cbs = None
            return

        def a(nbytes, stream, _user):
            try:
                return int(alloc(int(nbytes), stream or 0) or 0) or None
            except Exception:  # an allocator that raises has not served the request
                return None

        def f(ptr, nbytes, stream, _user):
            try:
                free(int(ptr or 0), int(nbytes), stream or 0)
            except Exception:
                pass

        cbs = (_lib.ALLOC_FN(a), _lib.FREE_FN(f))
        with self.lock:
            check(self._L.fmma_set_allocator(self._h, C.cast(cbs[0], C.c_void_p), C.cast(cbs[1], C.c_void_p), None))
        self._alloc_cbs = cbs  # the C library holds these function pointers

    def set_m2l_options(self, pair=-1, stages=0, group=0, units=0):
        """Tensor-core M2L switches: the 2-SM kernel (-1 default on, 0 off,
        1 on), the pipeline depth cap (0: as many as fit), the slots summed
        in TMEM between drains (0: default) and the (slot, K chunk) units per
        pipeline stage (0: by the expansion size)."""
        with self.lock:
            check(self._L.fmma_set_m2l_options(self._h, int(pair), int(stages), int(group), int(units)))

    def set_schedule_options(self, m2l_split=0, l2p_mode=0):
        """The plan autotuner's choices by hand: the slot split of small
        tensor-core M2L levels (0 fill the SMs, 1 none, 2 half, 3 double) and
        the leaf evaluation (0 by targets per leaf, 1 lanes over targets,
        2 lanes over coefficients)."""
        with self.lock:
            check(self._L.fmma_set_schedule_options(self._h, int(m2l_split), int(l2p_mode)))

    def debug_m2l_wait(self, wait_cycles=0, hold_issuer=False):
        """Test hook: the tensor-core M2L's wait bound in SM clocks (0: the
        default, ~2 s) and a hold of its MMA issuer on a flag that nothing
        sets, so the bound runs out and the solve raises status 5 (timeout)."""
        with self.lock:
            check(self._L.fmma_debug_m2l_wait(self._h, int(wait_cycles), 1 if hold_issuer else 0))

    def use_torch_allocator(self):
        """Takes the context's device memory from PyTorch's caching allocator
        (on the context's stream), so one memory budget serves both."""
        import torch
        dev = self.device

        def alloc(nbytes, stream):
            return torch.cuda.caching_allocator_alloc(nbytes, dev, stream)

        def free(ptr, nbytes, stream):
            torch.cuda.caching_allocator_delete(ptr)

        self.set_allocator(alloc, free)

    def _order(self, kind):
        """CUDA tensors are produced by work queued on torch's current stream;
        the context's own stream waits for that work (an event, no host
        block) before the library reads them.  Results are complete when a
        call returns (the library synchronises its stream)."""
        if kind != _lib.MEM_DEVICE:
            return
        import torch
        cur = torch.cuda.current_stream(self.device)
        if cur.cuda_stream == self.stream_ptr():
            return
        if self._xstream is None:
            self._xstream = torch.cuda.ExternalStream(self.stream_ptr(), device=f"cuda:{self.device}")
        ev = torch.cuda.Event()
        ev.record(cur)
        self._xstream.wait_event(ev)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.fmma_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_kernel(self, kernel, p0: float = 0.0):
        kid = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        check(self._L.fmma_set_kernel(self._h, kid, float(p0)))
        self.kernel = (kernel, p0)

    def set_kernel_expr(self, expr: str, translation_invariant: bool = False):
        """f(x, y) as a C++ expression in x[q], y[q], dx[q] = x[q] - y[q], r2 and
        r (double), compiled at run time for the device; e.g. "exp(-r2 / 0.01)".
        A compile error raises FmmaError with the compiler's log."""
        check(self._L.fmma_set_kernel_expr(self._h, str(expr).encode(), 1 if translation_invariant else 0))
        self.kernel = ("expr:" + str(expr), 0.0)

    # -- solve -------------------------------------------------------------
    def solve(self, tgt, src, w=None, *, solver="fmm", poly_ord=5, depth=-1, trans_sym=0,
              precision="fp64", out=None):
        """c[r, i] = sum_j w[r, j] f(tgt[i], src[j]).  Returns (ans, depth_used).

        tgt: (N, d), src: (M, d), w: None (unit weights), (M,) or (R, M);
        ans has shape (N,) or (R, N) and the dtype of the inputs.  For
        solver "nrnmm", depth is nrn_N (boxes per dimension, <= 0: default)
        and the second result is the nrn_N used."""
        t0 = tgt
        dtype = np.float64 if (t0.dtype == np.float64 or str(t0.dtype) == "torch.float64") else np.float32
        if tgt.ndim != 2 or src.ndim != 2 or tgt.shape[1] != src.shape[1]:
            raise ValueError("tgt and src must be (n, d) arrays of the same d")
        d = int(tgt.shape[1])
        nt, ns = int(tgt.shape[0]), int(src.shape[0])
        R = 1
        if w is not None:
            if w.ndim == 1:
                if w.shape[0] != ns:
                    raise ValueError("w must have one weight per source")
            elif w.ndim == 2:
                R = int(w.shape[0])
                if w.shape[1] != ns:
                    raise ValueError("w must be (R, n_src)")
            else:
                raise ValueError("w must be 1-D or 2-D")
        at, as_, aw = _Arr(tgt, dtype, "tgt"), _Arr(src, dtype, "src"), _Arr(w, dtype, "w")
        kind = _mem_kind(at, as_, aw)
        self._order(kind)
        if out is None:
            shape = (nt,) if (w is None or w.ndim == 1) else (R, nt)
            if kind == _lib.MEM_DEVICE:
                import torch
                out = torch.empty(shape, dtype=tgt.dtype, device=tgt.device)
            else:
                out = np.empty(shape, dtype=dtype)
        ao = _Arr(out, dtype, "out")
        if _mem_kind(at, ao) != kind:
            raise ValueError("out must live in the same memory as the inputs")
        used = C.c_int(0)
        fn = self._L.fmma_solve_d if dtype == np.float64 else self._L.fmma_solve_f
        with self.lock:
            check(fn(self._h, d, SOLVERS[solver], int(poly_ord), int(depth), int(trans_sym),
                     PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                     nt, at.ptr, ns, as_.ptr, R, aw.ptr, ao.ptr, kind, C.byref(used)))
        return out, used.value

    def solve_grad(self, tgt, src, w=None, *, solver="fmm", poly_ord=5, depth=-1, trans_sym=0,
                   precision="fp64", want_potential=True):
        """Potential c (optional) and its gradient with respect to the target
        positions, FP64.  Returns (c or None, grad, depth_used); grad has shape
        (N, d) or (R, N, d)."""
        d = int(tgt.shape[1])
        nt, ns = int(tgt.shape[0]), int(src.shape[0])
        R = 1 if (w is None or w.ndim == 1) else int(w.shape[0])
        at, as_, aw = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src"), _Arr(w, np.float64, "w")
        kind = _mem_kind(at, as_, aw)
        self._order(kind)
        single = w is None or w.ndim == 1
        pshape = (nt,) if single else (R, nt)
        gshape = (nt, d) if single else (R, nt, d)
        if kind == _lib.MEM_DEVICE:
            import torch
            pot = torch.empty(pshape, dtype=torch.float64, device=tgt.device) if want_potential else None
            grad = torch.empty(gshape, dtype=torch.float64, device=tgt.device)
            pp = pot.data_ptr() if pot is not None else None
            gp = grad.data_ptr()
        else:
            pot = np.empty(pshape) if want_potential else None
            grad = np.empty(gshape)
            pp = pot.ctypes.data if pot is not None else None
            gp = grad.ctypes.data
        used = C.c_int(0)
        with self.lock:
            check(self._L.fmma_solve_grad_d(self._h, d, SOLVERS[solver], int(poly_ord), int(depth), int(trans_sym),
                                            PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                                            nt, at.ptr, ns, as_.ptr, R, aw.ptr, pp, gp, kind, C.byref(used)))
        return pot, grad, used.value

    # -- forests of independent problems ------------------------------------
    def forest_depths(self, tgt, toff, src, soff, leaf_cap):
        """Per-problem Depth: smallest with at most leaf_cap points per leaf."""
        toff = np.ascontiguousarray(toff, dtype=np.int64)
        soff = np.ascontiguousarray(soff, dtype=np.int64)
        at, as_ = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src")
        kind = _mem_kind(at, as_)
        self._order(kind)
        nprob = len(toff) - 1
        out = np.zeros(nprob, dtype=np.int32)
        with self.lock:
            check(self._L.fmma_forest_depths_d(self._h, int(tgt.shape[1]), nprob, toff.ctypes.data_as(_lib._pi64),
                                               at.ptr, soff.ctypes.data_as(_lib._pi64), as_.ptr, int(leaf_cap), kind,
                                               out.ctypes.data_as(_lib._pi)))
        return out

    def forest_solve(self, tgt, toff, src, soff, w, depths, *, poly_ord=4, trans_sym=0, precision="fp64",
                     out=None):
        """All problems of a forest in one sweep.  tgt/src: concatenated (n, d)
        arrays with offsets toff/soff (nprob + 1 entries); w: (R, M) or (M,)."""
        toff = np.ascontiguousarray(toff, dtype=np.int64)
        soff = np.ascontiguousarray(soff, dtype=np.int64)
        depths = np.ascontiguousarray(depths, dtype=np.int32)
        nprob = len(toff) - 1
        d = int(tgt.shape[1])
        R = 1 if w.ndim == 1 else int(w.shape[0])
        at, as_, aw = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src"), _Arr(w, np.float64, "w")
        kind = _mem_kind(at, as_, aw)
        self._order(kind)
        nt = int(toff[-1])
        if out is None:
            shape = (nt,) if w.ndim == 1 else (R, nt)
            if kind == _lib.MEM_DEVICE:
                import torch
                out = torch.empty(shape, dtype=torch.float64, device=tgt.device)
            else:
                out = np.empty(shape)
        ao = _Arr(out, np.float64, "out")
        with self.lock:
            check(self._L.fmma_forest_solve_d(self._h, d, nprob, toff.ctypes.data_as(_lib._pi64), at.ptr,
                                              soff.ctypes.data_as(_lib._pi64), as_.ptr, R, aw.ptr, ao.ptr,
                                              int(poly_ord), depths.ctypes.data_as(_lib._pi), int(trans_sym),
                                              PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                                              kind))
        return out

    def plan(self, tgt, toff, src, soff, nrhs, depths, **kw) -> "Plan":
        return Plan(self, tgt, toff, src, soff, nrhs, depths, **kw)

    def set_tuner_cache(self, path: str):
        check(self._L.fmma_set_tuner_cache(self._h, path.encode()))

    def exact_rows(self, rows, tgt, src, w=None):
        """FP64 exact sum at the targets tgt[rows] (the sampled oracle)."""
        rows_a = rows
        R = 1 if (w is None or w.ndim == 1) else int(w.shape[0])
        d = int(tgt.shape[1])
        at, as_, aw = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src"), _Arr(w, np.float64, "w")
        kind = _mem_kind(at, as_, aw)
        self._order(kind)
        if kind == _lib.MEM_DEVICE:
            import torch
            rows_t = torch.as_tensor(rows_a, dtype=torch.int64, device=tgt.device).contiguous()
            out = torch.empty((R, rows_t.shape[0]), dtype=torch.float64, device=tgt.device)
            rp, op, nr = rows_t.data_ptr(), out.data_ptr(), int(rows_t.shape[0])
        else:
            rows_t = np.ascontiguousarray(rows_a, dtype=np.int64)
            out = np.empty((R, rows_t.shape[0]), dtype=np.float64)
            rp, op, nr = rows_t.ctypes.data, out.ctypes.data, int(rows_t.shape[0])
        with self.lock:
            check(self._L.fmma_exact_rows_d(self._h, d, nr, rp, int(tgt.shape[0]), at.ptr, int(src.shape[0]),
                                            as_.ptr, R, aw.ptr, op, kind))
        return out[0] if (w is None or w.ndim == 1) else out

    # -- global Chebyshev approximation (CHEBYSHEV_APPROX) --------------------
    def cheb_fit(self, values, dim: int, nth: int):
        """Coefficients of f ~ sum_i c_i prod_q T_{i_q}(x_q) on [-1, 1]^dim from
        f at the tensor nodes (cheb_points order).  values: ((nth+1)^dim,) or
        (nfunc, (nth+1)^dim), FP64; returns coefficients of the same shape."""
        size = (nth + 1) ** dim
        if values.shape[-1] != size or values.ndim not in (1, 2):
            raise ValueError("values must be ((nth+1)^dim,) or (nfunc, (nth+1)^dim)")
        nfunc = 1 if values.ndim == 1 else int(values.shape[0])
        av = _Arr(values, np.float64, "values")
        kind = _mem_kind(av)
        self._order(kind)
        if kind == _lib.MEM_DEVICE:
            import torch
            out = torch.empty(tuple(values.shape), dtype=torch.float64, device=values.device)
        else:
            out = np.empty(values.shape, dtype=np.float64)
        ao = _Arr(out, np.float64, "coef")
        with self.lock:
            check(self._L.fmma_cheb_fit_d(self._h, int(dim), int(nth), nfunc, av.ptr, ao.ptr, kind))
        return out

    def cheb_eval(self, coef, pts, nth: int):
        """sum_i coef[f, i] prod_q T_{i_q}(pts[p, q]) for every point (pts: (npts, dim)
        in [-1, 1]); shape (npts,) or (nfunc, npts)."""
        dim = int(pts.shape[1])
        size = (nth + 1) ** dim
        if coef.shape[-1] != size or coef.ndim not in (1, 2):
            raise ValueError("coef must be ((nth+1)^dim,) or (nfunc, (nth+1)^dim)")
        nfunc = 1 if coef.ndim == 1 else int(coef.shape[0])
        ac, ap = _Arr(coef, np.float64, "coef"), _Arr(pts, np.float64, "pts")
        kind = _mem_kind(ac, ap)
        self._order(kind)
        npts = int(pts.shape[0])
        shape = (npts,) if coef.ndim == 1 else (nfunc, npts)
        if kind == _lib.MEM_DEVICE:
            import torch
            out = torch.empty(shape, dtype=torch.float64, device=pts.device)
        else:
            out = np.empty(shape, dtype=np.float64)
        ao = _Arr(out, np.float64, "out")
        with self.lock:
            check(self._L.fmma_cheb_eval_d(self._h, dim, int(nth), nfunc, ac.ptr, npts, ap.ptr, ao.ptr, kind))
        return out

    # -- tree inspection -----------------------------------------------------
    def tree_export(self, tgt, src, depth):
        tgt = np.ascontiguousarray(tgt, dtype=np.float64)
        src = np.ascontiguousarray(src, dtype=np.float64)
        d = tgt.shape[1]
        tb = np.zeros(tgt.shape[0], dtype=np.int64)
        sb = np.zeros(src.shape[0], dtype=np.int64)
        ol = np.zeros(d + 1)
        with self.lock:
            check(self._L.fmma_tree_export_d(self._h, d, depth, tgt.shape[0], tgt.ctypes.data, src.shape[0],
                                             src.ctypes.data, tb.ctypes.data, sb.ctypes.data, ol.ctypes.data,
                                             _lib.MEM_HOST))
        return tb, sb, ol[:d].copy(), float(ol[d])

    def interaction_list(self, level, box):
        out = np.zeros(256, dtype=np.int64)
        cnt = C.c_int(0)
        with self.lock:
            check(self._L.fmma_interaction_list(self._h, level, box, out.ctypes.data_as(_lib._pi64), 256,
                                                C.byref(cnt)))
        return out[:cnt.value].copy()

    def near_list(self, box):
        out = np.zeros(32, dtype=np.int64)
        cnt = C.c_int(0)
        with self.lock:
            check(self._L.fmma_near_list(self._h, box, out.ctypes.data_as(_lib._pi64), 32, C.byref(cnt)))
        return out[:cnt.value].copy()

    def max_leaf_occupancy(self, tgt, src, depth):
        at, as_ = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src")
        kind = _mem_kind(at, as_)
        self._order(kind)
        mt, ms = C.c_int64(0), C.c_int64(0)
        with self.lock:
            check(self._L.fmma_max_leaf_occupancy_d(self._h, int(tgt.shape[1]), depth, int(tgt.shape[0]), at.ptr,
                                                    int(src.shape[0]), as_.ptr, kind, C.byref(mt), C.byref(ms)))
        return mt.value, ms.value

    # -- timing ----------------------------------------------------------------
    def stage_times(self) -> dict:
        ms = (C.c_double * _lib.NUM_STAGES)()
        check(self._L.fmma_stage_times(self._h, ms, _lib.NUM_STAGES))
        return {self._L.fmma_stage_name(i).decode(): ms[i] for i in range(_lib.NUM_STAGES)}

    def last_launch_count(self) -> int:
        return int(self._L.fmma_last_launch_count(self._h))

    def stream_ptr(self) -> int:
        """The context's cudaStream_t (for torch.cuda.ExternalStream)."""
        return int(self._L.fmma_ctx_stream(self._h) or 0)

    def m2l_stats(self) -> dict:
        ms, fl, n = C.c_double(0), C.c_double(0), C.c_int64(0)
        check(self._L.fmma_m2l_stats(self._h, C.byref(ms), C.byref(fl), C.byref(n)))
        return {"kernel_ms": ms.value, "flops": fl.value, "launches": n.value}

    def tree_stats(self) -> dict:
        a, b, c = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        check(self._L.fmma_tree_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"m2l_pairs": a.value, "p2p_pairs": b.value, "leaves": c.value}

    def tree_levels(self) -> dict:
        """Boxes and target rows per virtual level (0 = leaves) of the last fmm tree."""
        n = C.c_int(0)
        check(self._L.fmma_tree_levels(self._h, 0, C.byref(n), None, None))
        nb = np.zeros(n.value, dtype=np.int64)
        nr = np.zeros(n.value, dtype=np.int64)
        check(self._L.fmma_tree_levels(self._h, n.value, C.byref(n), nb.ctypes.data_as(C.c_void_p),
                                       nr.ctypes.data_as(C.c_void_p)))
        return {"boxes": nb.tolist(), "rows": nr.tolist()}


class Plan:
    """One geometry (a forest, or a single problem with toff = [0, n]), many
    weight sets: the sweep is captured in a CUDA graph and replayed."""

    def __init__(self, ctx: "Context", tgt, toff, src, soff, nrhs, depths, *, poly_ord=4, trans_sym=0,
                 precision="fp64", autotune=True):
        self._L = ctx._L
        toff = np.ascontiguousarray(toff, dtype=np.int64)
        soff = np.ascontiguousarray(soff, dtype=np.int64)
        depths = np.ascontiguousarray(depths, dtype=np.int32)
        at, as_ = _Arr(tgt, np.float64, "tgt"), _Arr(src, np.float64, "src")
        kind = _mem_kind(at, as_)
        ctx._order(kind)
        self._ctx = ctx
        self.nt, self.ns, self.nrhs, self.d = int(toff[-1]), int(soff[-1]), int(nrhs), int(tgt.shape[1])
        h = C.c_void_p()
        with ctx.lock:
            check(self._L.fmma_plan_create_d(ctx.handle, self.d, len(toff) - 1, toff.ctypes.data_as(_lib._pi64),
                                             at.ptr, soff.ctypes.data_as(_lib._pi64), as_.ptr, self.nrhs,
                                             int(poly_ord), depths.ctypes.data_as(_lib._pi), int(trans_sym),
                                             PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                                             1 if autotune else 0, kind, C.byref(h)))
        self._h = h

    def execute(self, w, out=None):
        aw = _Arr(w, np.float64, "w")
        shape = (self.nt,) if w.ndim == 1 else (self.nrhs, self.nt)
        if out is None:
            if aw.kind == _lib.MEM_DEVICE:
                import torch
                out = torch.empty(shape, dtype=torch.float64, device=w.device)
            else:
                out = np.empty(shape)
        ao = _Arr(out, np.float64, "out")
        self._ctx._order(aw.kind)
        check(self._L.fmma_plan_execute_d(self._h, aw.ptr, ao.ptr, aw.kind))
        return out

    def stats(self) -> dict:
        b, e = C.c_double(0), C.c_double(0)
        tc, f64, nodes = C.c_int(0), C.c_int(0), C.c_int64(0)
        check(self._L.fmma_plan_stats(self._h, C.byref(b), C.byref(e), C.byref(tc), C.byref(f64), C.byref(nodes)))
        return {"build_ms": b.value, "last_exec_ms": e.value, "levels_tc": tc.value, "levels_fp64": f64.value,
                "graph_nodes": nodes.value}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.fmma_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}
_default_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    """A process-wide context per device (shared operator cache)."""
    with _default_lock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


def choose_depth(ctx: Context, tgt, src, cap: int, start: int = 2, limit: int = 22) -> int:
    """Smallest Depth whose largest leaf holds at most `cap` targets and at
    most `cap` sources."""
    for L in range(start, limit + 1):
        mt, ms = ctx.max_leaf_occupancy(tgt, src, L)
        if mt <= cap and ms <= cap:
            return L
    raise ValueError(f"no depth <= {limit} meets the leaf cap {cap}")


def version() -> str:
    return _lib.load().fmma_version().decode()


def cheb_nodes(nth: int) -> np.ndarray:
    """The 1-D Chebyshev nodes cos((2k+1) pi / (2 nth + 2)), k = 0..nth."""
    out = np.zeros(nth + 1)
    L = _lib.load()
    st = L.fmma_cheb_nodes(int(nth), out.ctypes.data_as(_lib._pd))
    if st != 0:
        raise FmmaError(st, L.fmma_last_error().decode())
    return out


def cheb_points(dim: int, nth: int) -> np.ndarray:
    """The (nth+1)^dim fit points of cheb_fit, (size, dim), dimension 0 fastest
    (the node order of the reference's CHEBYSHEV_APPROX::initialize)."""
    x = cheb_nodes(nth)
    n = nth + 1
    idx = np.arange(n ** dim)
    return np.stack([x[(idx // n ** q) % n] for q in range(dim)], axis=1)
