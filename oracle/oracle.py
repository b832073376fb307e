"""ctypes bindings of the CPU oracle (oracle/_build/liboracle.so) and of the
compiled reference (oracle/_ref/libfmma_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg.  The product path never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfmma_ref.so")

_i64 = C.c_int64
_pd = C.POINTER(C.c_double)
_pf = C.POINTER(C.c_float)
_pi64 = C.POINTER(C.c_int64)


def reference_dir() -> str | None:
    """The reference source tree: $FMMA_REFERENCE_DIR, else a directory named
    `reference` beside this repository; None when neither holds src/fmm.cpp."""
    for d in (os.environ.get("FMMA_REFERENCE_DIR"),
              os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if d and os.path.isfile(os.path.join(d, "src", "fmm.cpp")):
            return os.path.abspath(d)
    return None


def build(ref_root: str | None = None) -> None:
    """Compiles the oracle and, when the reference tree exists, the reference."""
    ref_root = ref_root or reference_dir()
    args = ["make", "-s", "-C", HERE, f"REF={ref_root or '/nonexistent'}"]
    subprocess.check_call(args, env=dict(os.environ))


def _dp(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _fp(a):
    return None if a is None else a.ctypes.data_as(_pf)


class Oracle:
    """The C restatement of the reference's exact, fmm, tree and nrnmm solvers."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        L = C.CDLL(path)
        L.orc_exact.argtypes = [C.c_int, C.c_int, C.c_double, _i64, _pd, _i64, _pd, _pd, _pd]
        L.orc_exact_rows.argtypes = [C.c_int, C.c_int, C.c_double, _i64, _pi64, _pd, _i64, _pd, _pd, _pd]
        L.orc_fmm.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                              _i64, _pd, _i64, _pd, _pd, _pd]
        L.orc_fmm.restype = C.c_int
        L.orc_tree.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                               _i64, _pd, _i64, _pd, _pd, _pd]
        L.orc_tree.restype = C.c_int
        L.orc_nrnmm.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                _i64, _pd, _i64, _pd, _pd, _pd]
        L.orc_nrnmm.restype = C.c_int
        L.orc_default_nrn.argtypes = [_i64, C.c_int]
        L.orc_default_nrn.restype = C.c_int
        L.orc_cheb_fit.argtypes = [C.c_int, C.c_int, _pd, _pd]
        L.orc_cheb_fit.restype = C.c_int
        L.orc_cheb_eval.argtypes = [C.c_int, C.c_int, _pd, _i64, _pd, _pd]
        L.orc_default_depth.argtypes = [_i64, C.c_int]
        L.orc_default_depth.restype = C.c_int
        L.orc_origin_len.argtypes = [C.c_int, _i64, _pd, _i64, _pd, _pd, _pd]
        L.orc_bin_points.argtypes = [C.c_int, C.c_int, _i64, _pd, _pd, C.c_double, _pi64]
        L.orc_far_list_rowmajor.argtypes = [C.c_int, _i64, C.c_int, _pi64]
        L.orc_far_list_rowmajor.restype = C.c_int
        L.orc_near_list_rowmajor.argtypes = [C.c_int, _i64, C.c_int, _pi64]
        L.orc_near_list_rowmajor.restype = C.c_int
        L.orc_chebyshev.argtypes = [C.c_int, C.c_double]
        L.orc_chebyshev.restype = C.c_double
        L.orc_schebyshev.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_schebyshev.restype = C.c_double
        self.L = L

    @staticmethod
    def _pts(x, d):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, d)
        return x

    def exact(self, d, kid, p0, tgt, src, w=None):
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(t.shape[0])
        self.L.orc_exact(d, kid, p0, t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(w), _dp(out))
        return out

    def exact_rows(self, d, kid, p0, rows, tgt, src, w=None):
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(rows.shape[0])
        self.L.orc_exact_rows(d, kid, p0, rows.shape[0], rows.ctypes.data_as(_pi64), _dp(t),
                              s.shape[0], _dp(s), _dp(w), _dp(out))
        return out

    def fmm(self, d, kid, p0, poly_ord, depth, trans_sym, tgt, src, w=None):
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(t.shape[0])
        used = self.L.orc_fmm(d, kid, p0, poly_ord, depth, trans_sym, t.shape[0], _dp(t),
                              s.shape[0], _dp(s), _dp(w), _dp(out))
        if used < 0:
            raise ValueError("oracle: unsupported size")
        return out, used

    def tree(self, d, kid, p0, poly_ord, depth, tgt, src, w=None):
        """The reference's tree solver (src/tree.cpp:12-100)."""
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(t.shape[0])
        used = self.L.orc_tree(d, kid, p0, poly_ord, depth, t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(w), _dp(out))
        if used < 0:
            raise ValueError("oracle: unsupported size")
        return out, used

    def nrnmm(self, d, kid, p0, poly_ord, nrn, tgt, src, w=None):
        """The reference's nrnmm solver (src/nrnmm.cpp:13-102); returns (ans, nrn used)."""
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(t.shape[0])
        used = self.L.orc_nrnmm(d, kid, p0, poly_ord, nrn, t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(w), _dp(out))
        if used < 0:
            raise ValueError("oracle: unsupported size")
        return out, used

    def cheb_fit(self, dim, nth, values):
        """Coefficients of the reference's collocation system, solved directly."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        coef = np.zeros(v.shape[0])
        if self.L.orc_cheb_fit(dim, nth, _dp(v), _dp(coef)) < 0:
            raise ValueError("oracle: unsupported size")
        return coef

    def cheb_eval(self, dim, nth, coef, pts):
        """The reference's predict at every point (NaN outside [-1, 1])."""
        c = np.ascontiguousarray(coef, dtype=np.float64)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, dim)
        out = np.zeros(p.shape[0])
        self.L.orc_cheb_eval(dim, nth, _dp(c), p.shape[0], _dp(p), _dp(out))
        return out

    def default_nrn(self, ns, d):
        return self.L.orc_default_nrn(ns, d)

    def default_depth(self, nt, d):
        return self.L.orc_default_depth(nt, d)

    def origin_len(self, d, tgt, src):
        t = self._pts(tgt, d)
        s = self._pts(src, d)
        o = np.zeros(d)
        L = C.c_double()
        self.L.orc_origin_len(d, t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(o), C.byref(L))
        return o, L.value

    def bin_points(self, d, depth, x, origin, Len):
        x = self._pts(x, d)
        o = np.ascontiguousarray(origin, dtype=np.float64)
        out = np.zeros(x.shape[0], dtype=np.int64)
        self.L.orc_bin_points(d, depth, x.shape[0], _dp(x), _dp(o), Len, out.ctypes.data_as(_pi64))
        return out

    def far_list(self, d, box, N):
        out = np.zeros(256, dtype=np.int64)
        n = self.L.orc_far_list_rowmajor(d, box, N, out.ctypes.data_as(_pi64))
        return out[:n].copy()

    def near_list(self, d, box, N):
        out = np.zeros(32, dtype=np.int64)
        n = self.L.orc_near_list_rowmajor(d, box, N, out.ctypes.data_as(_pi64))
        return out[:n].copy()

    def chebyshev(self, n, x):
        return self.L.orc_chebyshev(n, x)

    def schebyshev(self, n, x, y):
        return self.L.orc_schebyshev(n, x, y)


class Reference:
    """The reference library compiled from its own sources (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"compiled reference missing: {path}")
        L = C.CDLL(path)
        L.ref_solve_d.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int,
                                  C.c_int, _i64, _pd, _i64, _pd, _pd, _pd]
        L.ref_solve_d.restype = C.c_int
        L.ref_solve_f.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int,
                                  C.c_int, _i64, _pf, _i64, _pf, _pf, _pf]
        L.ref_solve_f.restype = C.c_int
        L.ref_p2m_d.argtypes = [C.c_int, C.c_int, C.c_int, _i64, _pd, _i64, _pd, _pd, _pi64, _pd, _pd]
        L.ref_p2m_f.argtypes = [C.c_int, C.c_int, C.c_int, _i64, _pf, _i64, _pf, _pf, _pi64, _pf]
        L.ref_chebyshev.argtypes = [C.c_int, C.c_double]
        L.ref_chebyshev.restype = C.c_double
        L.ref_schebyshev.argtypes = [C.c_int, C.c_double, C.c_double]
        L.ref_schebyshev.restype = C.c_double
        L.ref_num_threads.restype = C.c_int
        L.ref_cheb_fit_d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _pd, _pd]
        L.ref_cheb_predict_d.argtypes = [C.c_int, C.c_int, _pd, _i64, _pd, _pd]
        self.L = L

    def solve(self, d, solver, kid, p0, poly_ord, depth, trans_sym, tgt, src, w=None,
              dtype=np.float64):
        t = np.ascontiguousarray(tgt, dtype=dtype).reshape(-1, d)
        s = np.ascontiguousarray(src, dtype=dtype).reshape(-1, d)
        w = None if w is None else np.ascontiguousarray(w, dtype=dtype)
        out = np.zeros(t.shape[0], dtype=dtype)
        if dtype == np.float64:
            used = self.L.ref_solve_d(d, solver.encode(), kid, p0, poly_ord, depth, trans_sym,
                                      t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(w), _dp(out))
        else:
            used = self.L.ref_solve_f(d, solver.encode(), kid, p0, poly_ord, depth, trans_sym,
                                      t.shape[0], _fp(t), s.shape[0], _fp(s), _fp(w), _fp(out))
        return out, used

    def p2m_bins(self, d, depth, poly_ord, tgt, src, w, dtype=np.float64, want_wm=False):
        t = np.ascontiguousarray(tgt, dtype=dtype).reshape(-1, d)
        s = np.ascontiguousarray(src, dtype=dtype).reshape(-1, d)
        w = np.ascontiguousarray(w, dtype=dtype)
        box = np.full(s.shape[0], -1, dtype=np.int64)
        ol = np.zeros(d + 1, dtype=dtype)
        if dtype == np.float64:
            wm = None
            if want_wm:
                nb = (1 << (depth - 1)) ** d
                wm = np.zeros(nb * (poly_ord + 1) ** d)
            self.L.ref_p2m_d(d, depth, poly_ord, t.shape[0], _dp(t), s.shape[0], _dp(s), _dp(w),
                             box.ctypes.data_as(_pi64), _dp(ol), _dp(wm))
            return box, ol, wm
        self.L.ref_p2m_f(d, depth, poly_ord, t.shape[0], _fp(t), s.shape[0], _fp(s), _fp(w),
                         box.ctypes.data_as(_pi64), _fp(ol))
        return box, ol, None

    def cheb_fit(self, dim, nth, fid, a=0, b=0):
        """CHEBYSHEV_APPROX<double, dim>::initialize on test function fid:
        (values at the nodes, coefficients), both in the reference's order."""
        size = (nth + 1) ** dim
        values, coef = np.zeros(size), np.zeros(size)
        self.L.ref_cheb_fit_d(dim, nth, fid, a, b, _dp(values), _dp(coef))
        return values, coef

    def cheb_predict(self, dim, nth, coef, pts):
        c = np.ascontiguousarray(coef, dtype=np.float64)
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, dim)
        out = np.zeros(p.shape[0])
        self.L.ref_cheb_predict_d(dim, nth, _dp(c), p.shape[0], _dp(p), _dp(out))
        return out

    def num_threads(self):
        return self.L.ref_num_threads()
