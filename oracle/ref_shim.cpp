// ref_shim.cpp — C entry points over the compiled reference (fockl/FMMA).
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's own sources (src/*.cpp, read where they lie) into
// oracle/_ref/libfmma_ref.so.  Tests use it to pin the oracle restatement and
// to make golden vectors; the benchmark's reference arm times it on the host
// cores.  Nothing in the product path links it.
//
// The kernels below are the reference-side spellings of the built-in kernel
// ids of include/fmma_b200.h, passed to the reference through its own
// FMMA::set_fn (include/fmma/fmma.hpp:79-82).
#include <array>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fmma/chebyshev_approx.hpp"
#include "fmma/fmma.hpp"
#include "fmma/math.hpp"
#include "../include/fmma_b200.h"

namespace {

template <typename T, std::size_t D>
std::function<T(const std::array<T, D>&, const std::array<T, D>&)> make_fn(int kid, double p0) {
  using A = std::array<T, D>;
  switch (kid) {
    case FMMA_KERNEL_INV_R:
      return [](const A& x, const A& y) {
        double r2 = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; }
        return (T)(1.0 / std::sqrt(r2));
      };
    case FMMA_KERNEL_INV_R_SAFE:
      return [](const A& x, const A& y) {
        double r2 = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; }
        return (T)(r2 > 0.0 ? 1.0 / std::sqrt(r2) : 0.0);
      };
    case FMMA_KERNEL_INV_DIFF:
      return [](const A& x, const A& y) {
        double t = x[0] - y[0];
        return (T)(t != 0.0 ? 1.0 / t : 0.0);
      };
    case FMMA_KERNEL_LOG_R:
      return [](const A& x, const A& y) {
        double r2 = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; }
        return (T)(r2 > 0.0 ? 0.5 * std::log(r2) : 0.0);
      };
    case FMMA_KERNEL_GAUSSIAN:
      return [p0](const A& x, const A& y) {
        double r2 = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; }
        return (T)std::exp(-r2 / p0);
      };
    case FMMA_KERNEL_MULTIQUADRIC:
      return [p0](const A& x, const A& y) {
        double r2 = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; }
        return (T)std::sqrt(r2 + p0);
      };
    case FMMA_KERNEL_SUM_OVER_R2:
      return [](const A& x, const A& y) {
        double r2 = 0.0, s = 0.0;
        for (std::size_t k = 0; k < D; ++k) { double t = x[k] - y[k]; r2 += t * t; s += t; }
        return (T)(s / r2);
      };
    case FMMA_KERNEL_SUM2_OVER_R2:
    default:
      return [](const A& x, const A& y) {
        double r2 = 0.0, s = 0.0;
        for (std::size_t k = 0; k < D; ++k) {
          double t = x[k] - y[k], u = x[k] + y[k];
          r2 += t * t; s += u * u;
        }
        return (T)(s / r2);
      };
  }
}

template <typename T, std::size_t D>
std::vector<std::array<T, D>> to_points(int64_t n, const T* p) {
  std::vector<std::array<T, D>> v((std::size_t)n);
  for (int64_t i = 0; i < n; ++i)
    for (std::size_t k = 0; k < D; ++k) v[(std::size_t)i][k] = p[i * (int64_t)D + (int64_t)k];
  return v;
}

// Exposes the protected stage methods, the way test/src/fmma/m2m.cpp does.
template <typename T, std::size_t D>
class Probe : public fmma::FMMA<T, D> {
 public:
  void origin_len(const std::vector<std::array<T, D>>& a, const std::vector<std::array<T, D>>& b,
                  T* origin, T* Len) {
    std::array<T, D> o;
    T L;
    this->get_origin_and_length(a, b, o, L);
    for (std::size_t k = 0; k < D; ++k) origin[k] = o[k];
    *Len = L;
  }
  void p2m(const std::vector<T>& w, const std::vector<std::array<T, D>>& s, int N,
           const std::array<T, D>& origin, T len, std::vector<std::vector<std::size_t>>& lists,
           std::vector<std::vector<T>>& Wm) {
    std::vector<std::array<T, D>> nodes;
    this->P2M(w, s, N, origin, len, lists, Wm, nodes);
  }
};

template <typename T, std::size_t D>
int solve_t(const char* solver, int kid, double p0, int poly_ord, int depth, int trans_sym,
            int64_t nt, const T* tgt, int64_t ns, const T* src, const T* w, T* ans) {
  fmma::FMMA<T, D> f;
  f.set_fn(make_fn<T, D>(kid, p0));
  f.set_solver_type(solver);
  f.set_poly_ord(poly_ord);
  f.set_Depth(depth);
  f.set_trans_sym_flag(trans_sym);
  const bool nrnmm = std::string(solver) == "nrnmm";
  if (nrnmm) f.set_nrn_N(depth);  // the depth slot carries nrn_N for this solver
  auto t = to_points<T, D>(nt, tgt);
  auto s = to_points<T, D>(ns, src);
  std::vector<T> a((std::size_t)nt, (T)0);
  if (w) {
    std::vector<T> wv(w, w + ns);
    f.solve(t, wv, s, a);
  } else {
    f.solve(t, s, a);
  }
  for (int64_t i = 0; i < nt; ++i) ans[i] = a[(std::size_t)i];
  if (depth > 0) return depth;
  if (nrnmm) return (int)(std::sqrt(3.0) * std::pow((T)ns, 1.0 / (2.0 * D))) + 1;  // src/nrnmm.cpp:20-22
  int D_ = (int)(std::log((double)nt) / (double)D) + 1;
  return D_ <= 0 ? 1 : D_;
}

template <typename T, std::size_t D>
void bins_t(int depth, int64_t nt, const T* tgt, int64_t ns, const T* src, const T* w,
            int poly_ord, int64_t* src_box, T* origin_len, T* wm_leaf) {
  Probe<T, D> p;
  p.set_poly_ord(poly_ord);
  auto t = to_points<T, D>(nt, tgt);
  auto s = to_points<T, D>(ns, src);
  T o[3], L;
  p.origin_len(t, s, o, &L);
  std::array<T, D> oa;
  for (std::size_t k = 0; k < D; ++k) { oa[k] = o[k]; origin_len[k] = o[k]; }
  origin_len[D] = L;
  int N = 1 << (depth - 1);
  std::vector<std::vector<std::size_t>> lists;
  std::vector<std::vector<T>> Wm;
  std::vector<T> wv(w, w + ns);
  p.p2m(wv, s, N, oa, L / N, lists, Wm);
  for (std::size_t b = 0; b < lists.size(); ++b)
    for (auto i : lists[b]) src_box[i] = (int64_t)b;
  if (wm_leaf) {
    std::size_t P = Wm.empty() ? 0 : Wm[0].size();
    for (std::size_t b = 0; b < Wm.size(); ++b)
      for (std::size_t k = 0; k < P; ++k) wm_leaf[b * P + k] = Wm[b][k];
  }
}

// Test functions for the Chebyshev approximation: 0 = |x|^2 (the class's
// default fn), 1 = 1 / (1 + |x|^2) (test/src/chebyshev_approx/common.cpp:
// 166-170), 2 = exp(x_0) cos(2 x_{D-1}), 3 = T_a(x_0) T_b(x_1) written out as
// the reference's coefficient tests do (:11-25).
template <typename T, std::size_t D>
std::function<T(const std::array<T, D>&)> cheb_fn(int fid, int a, int b) {
  return [=](const std::array<T, D>& x) -> T {
    double len2 = 0.0;
    for (std::size_t q = 0; q < D; ++q) len2 += x[q] * x[q];
    auto tk = [](int k, double v) { return k == 0 ? 1.0 : (k == 1 ? v : (k == 2 ? 2 * v * v - 1 : 4 * v * v * v - 3 * v)); };
    switch (fid) {
      case 0: return (T)len2;
      case 1: return (T)(1.0 / (1.0 + len2));
      case 2: return (T)(std::exp((double)x[0]) * std::cos(2.0 * x[D - 1]));
      default: return (T)(tk(a, x[0]) * (D > 1 ? tk(b, x[1]) : 1.0));
    }
  };
}

template <typename T, std::size_t D>
void cheb_fit_t(int nth, int fid, int a, int b, double* values, double* coef) {
  fmma::CHEBYSHEV_APPROX<T, D> c;
  c.fn = cheb_fn<T, D>(fid, a, b);
  c.Nth = nth;
  std::srand(0);  // the GCR start is drawn with rand()
  c.initialize();
  const int n = nth + 1;
  for (std::size_t i = 0; i < c.size; ++i) {
    std::array<T, D> pos;
    std::size_t ic = i;
    for (std::size_t q = 0; q < D; ++q) {  // the node order of initialize (src/chebyshev_approx.cpp:50-55)
      pos[q] = (T)std::cos((2.0 * (ic % n) + 1.0) / (2 * nth + 2) * M_PI);
      ic /= n;
    }
    values[i] = (double)c.fn(pos);
    coef[i] = (double)c.coef[i];
  }
}

template <typename T, std::size_t D>
void cheb_predict_t(int nth, const double* coef, int64_t npts, const double* pts, double* out) {
  fmma::CHEBYSHEV_APPROX<T, D> c;
  c.Nth = nth;
  c.size = 1;
  for (std::size_t q = 0; q < D; ++q) c.size *= nth + 1;
  c.coef.assign(coef, coef + c.size);
  for (int64_t p = 0; p < npts; ++p) {
    std::array<T, D> pos;
    for (std::size_t q = 0; q < D; ++q) pos[q] = (T)pts[p * D + q];
    out[p] = (double)c.predict(pos);
  }
}

}  // namespace

extern "C" {

// CHEBYSHEV_APPROX<double, dim>: the function values at the nodes and the
// fitted coefficients ((nth+1)^dim each, the reference's order).
void ref_cheb_fit_d(int dim, int nth, int fid, int a, int b, double* values, double* coef) {
  switch (dim) {
    case 1: cheb_fit_t<double, 1>(nth, fid, a, b, values, coef); break;
    case 2: cheb_fit_t<double, 2>(nth, fid, a, b, values, coef); break;
    case 3: cheb_fit_t<double, 3>(nth, fid, a, b, values, coef); break;
  }
}

// CHEBYSHEV_APPROX<double, dim>::predict with the given coefficients.
void ref_cheb_predict_d(int dim, int nth, const double* coef, int64_t npts, const double* pts, double* out) {
  switch (dim) {
    case 1: cheb_predict_t<double, 1>(nth, coef, npts, pts, out); break;
    case 2: cheb_predict_t<double, 2>(nth, coef, npts, pts, out); break;
    case 3: cheb_predict_t<double, 3>(nth, coef, npts, pts, out); break;
  }
}


// Runs FMMA<double,dim>::solve with solver "exact" or "fmm" (or any other
// solver name the reference knows).  Returns the depth used.
int ref_solve_d(int dim, const char* solver, int kid, double p0, int poly_ord, int depth,
                int trans_sym, int64_t nt, const double* tgt, int64_t ns, const double* src,
                const double* w, double* ans) {
  switch (dim) {
    case 1: return solve_t<double, 1>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
    case 2: return solve_t<double, 2>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
    case 3: return solve_t<double, 3>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
  }
  return -1;
}

int ref_solve_f(int dim, const char* solver, int kid, double p0, int poly_ord, int depth,
                int trans_sym, int64_t nt, const float* tgt, int64_t ns, const float* src,
                const float* w, float* ans) {
  switch (dim) {
    case 1: return solve_t<float, 1>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
    case 2: return solve_t<float, 2>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
    case 3: return solve_t<float, 3>(solver, kid, p0, poly_ord, depth, trans_sym, nt, tgt, ns, src, w, ans);
  }
  return -1;
}

// Leaf box (row-major) of every source as the reference's P2M lists it, the
// cube origin/Len, and the leaf multipole coefficients (dense grid, P each).
void ref_p2m_d(int dim, int depth, int poly_ord, int64_t nt, const double* tgt, int64_t ns,
               const double* src, const double* w, int64_t* src_box, double* origin_len,
               double* wm_leaf) {
  switch (dim) {
    case 1: bins_t<double, 1>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, wm_leaf); break;
    case 2: bins_t<double, 2>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, wm_leaf); break;
    case 3: bins_t<double, 3>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, wm_leaf); break;
  }
}

void ref_p2m_f(int dim, int depth, int poly_ord, int64_t nt, const float* tgt, int64_t ns,
               const float* src, const float* w, int64_t* src_box, float* origin_len) {
  switch (dim) {
    case 1: bins_t<float, 1>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, nullptr); break;
    case 2: bins_t<float, 2>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, nullptr); break;
    case 3: bins_t<float, 3>(depth, nt, tgt, ns, src, w, poly_ord, src_box, origin_len, nullptr); break;
  }
}

double ref_chebyshev(int n, double x) { return fmma::Chebyshev(n, x); }
double ref_schebyshev(int n, double x, double y) { return fmma::SChebyshev(n, x, y); }

int ref_num_threads(void) {
#ifdef _OPENMP
  int n = 1;
#pragma omp parallel
  {
#pragma omp single
    n = omp_get_num_threads();
  }
  return n;
#else
  return 1;
#endif
}

}  // extern "C"
