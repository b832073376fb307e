// fmma/fmma.hpp — header-only drop-in for fockl/FMMA's fmma::FMMA<TYPE,DIM>
// (reference include/fmma/fmma.hpp:52-170), running the `exact`, `fmm`,
// `tree` and `nrnmm` solvers on a B200 through the C ABI of fmma_b200.h.
//
// Kept: the class template, the std::array arithmetic helpers, the setters
// (set_fn/set_fn1/set_fn2, set_solver_type, set_nrn_N, set_poly_ord,
// set_Depth, set_trans_sym_flag), check_blas, both solve overloads, the
// per-solver methods, the sticky default Depth, the time log and the
// reference's error behaviour (message on stderr, exit(EXIT_FAILURE)) unless
// exceptions are switched on with set_throw_on_error(true).
//
// Kernels: built-in device functors from fmma::kernels, or any __device__
// functor through set_fn_device (include/fmma/device.cuh, nvcc only).  A
// host std::function cannot run on the device; those overloads report an
// error instead of falling back to the CPU.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../fmma_b200.h"

namespace fmma {

// std::array helpers (reference include/fmma/fmma.hpp:15-49)
template <typename TYPE, std::size_t DIM>
std::array<TYPE, DIM> operator+(const std::array<TYPE, DIM>& a, const std::array<TYPE, DIM>& b) {
  std::array<TYPE, DIM> r;
  for (std::size_t d = 0; d < DIM; ++d) r[d] = a[d] + b[d];
  return r;
}
template <typename TYPE, std::size_t DIM>
std::array<TYPE, DIM> operator-(const std::array<TYPE, DIM>& a, const std::array<TYPE, DIM>& b) {
  std::array<TYPE, DIM> r;
  for (std::size_t d = 0; d < DIM; ++d) r[d] = a[d] - b[d];
  return r;
}
template <typename TYPE, std::size_t DIM>
std::array<TYPE, DIM> operator*(const std::array<TYPE, DIM>& a, const std::array<TYPE, DIM>& b) {
  std::array<TYPE, DIM> r;
  for (std::size_t d = 0; d < DIM; ++d) r[d] = a[d] * b[d];
  return r;
}
template <typename TYPE, std::size_t DIM>
std::array<TYPE, DIM> operator/(const std::array<TYPE, DIM>& a, const std::array<TYPE, DIM>& b) {
  std::array<TYPE, DIM> r;
  for (std::size_t d = 0; d < DIM; ++d) r[d] = a[d] / b[d];
  return r;
}

// Built-in interaction kernels (device functors of libfmma_b200).
namespace kernels {
struct Kernel {
  int id;
  double p0;
};
inline Kernel inv_r() { return {FMMA_KERNEL_INV_R, 0.0}; }        // 1/|x-y| (reference default)
inline Kernel laplace() { return {FMMA_KERNEL_INV_R_SAFE, 0.0}; }  // 1/|x-y|, 0 at coincidence
inline Kernel inv_diff() { return {FMMA_KERNEL_INV_DIFF, 0.0}; }   // 1/(x-y), 1-D
inline Kernel log_r() { return {FMMA_KERNEL_LOG_R, 0.0}; }         // log|x-y|, 0 at coincidence
inline Kernel gaussian(double p0 = 0.01) { return {FMMA_KERNEL_GAUSSIAN, p0}; }
inline Kernel multiquadric(double p0 = 1e-4) { return {FMMA_KERNEL_MULTIQUADRIC, p0}; }
inline Kernel sum_over_r2() { return {FMMA_KERNEL_SUM_OVER_R2, 0.0}; }
inline Kernel sum2_over_r2() { return {FMMA_KERNEL_SUM2_OVER_R2, 0.0}; }
}  // namespace kernels

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

template <typename TYPE, std::size_t DIM>
class FMMA {
  static_assert(std::is_same<TYPE, double>::value || std::is_same<TYPE, float>::value, "TYPE is float or double");
  static_assert(DIM >= 1 && DIM <= 3, "DIM is 1, 2 or 3");

 public:
  using point = std::array<TYPE, DIM>;

  // The reference's functor member (include/fmma/fmma.hpp:55-63); kept for
  // source compatibility only, it is never evaluated.
  std::function<TYPE(const point&, const point&)> fn;

  FMMA() = default;
  ~FMMA() {
    if (ctx_) fmma_ctx_destroy(ctx_);
  }
  FMMA(const FMMA&) = delete;
  FMMA& operator=(const FMMA&) = delete;

  // ---- kernels ------------------------------------------------------------
  void set_fn(kernels::Kernel k) {
    kernel_ = k;
    user_hook_ = nullptr;
    user_obj_.reset();
    expr_ = false;
  }
  // f as a C++ expression compiled at run time (fmma_set_kernel_expr): in
  // x[q], y[q], dx[q] = x[q] - y[q], r2 = |x - y|^2, r = |x - y|.  A kernel of
  // the difference alone (the reference's set_fn1) is translation invariant.
  void set_fn_expr(const std::string& expr, bool translation_invariant = false) {
    user_hook_ = nullptr;
    user_obj_.reset();
    expr_ = false;
    check(fmma_set_kernel_expr(context(), expr.c_str(), translation_invariant ? 1 : 0));
    expr_ = true;
  }
  void set_fn1(kernels::Kernel k) { set_fn(k); }
  void set_fn2(kernels::Kernel k) { set_fn(k); }
  void set_fn(const std::function<TYPE(const point&)>&) { host_functor(); }
  void set_fn1(const std::function<TYPE(const point&)>&) { host_functor(); }
  void set_fn(const std::function<TYPE(const point&, const point&)>&) { host_functor(); }
  void set_fn2(const std::function<TYPE(const point&, const point&)>&) { host_functor(); }
#ifdef __CUDACC__
  // Any __device__ functor f(const std::array<double,DIM>& x, const
  // std::array<double,DIM>& y) -> double; defined in fmma/device.cuh.
  template <class F>
  void set_fn_device(F f, bool translation_invariant = true);
#endif

  // ---- parameters (include/fmma/fmma.hpp:88-127) ----------------------------
  void set_solver_type(const std::string new_type) { solver_type_ = new_type; }
  void set_nrn_N(int n) { nrn_N_ = n; }
  void set_poly_ord(int p) { poly_ord_ = p; }
  void set_Depth(int d) { Depth_ = d; }
  void set_trans_sym_flag(int f) { trans_sym_flag_ = f; }
  // extensions
  void set_precision(int p) { precision_ = p; }  // FMMA_PREC_FP64 / _MIXED_TF32X3 / _MIXED_BF16X3
  void set_device(int d) { device_ = d; }
  void set_throw_on_error(bool t) { throw_ = t; }
  int get_Depth() const { return Depth_; }
  int get_nrn_N() const { return nrn_N_; }

  bool check_blas(void) { return false; }

  // ---- solve (src/fmma.cpp:143-207) ---------------------------------------
  void solve(const std::vector<point>& target, const std::vector<point>& source, std::vector<TYPE>& ans) {
    run(solver_type_, target, nullptr, source, ans);
  }
  void solve(const std::vector<point>& target, const std::vector<TYPE>& source_weight,
             const std::vector<point>& source, std::vector<TYPE>& ans) {
    run(solver_type_, target, &source_weight, source, ans);
  }
  void exact(const std::vector<point>& t, const std::vector<point>& s, std::vector<TYPE>& a) { run("exact", t, nullptr, s, a); }
  void exact(const std::vector<point>& t, const std::vector<TYPE>& w, const std::vector<point>& s, std::vector<TYPE>& a) {
    run("exact", t, &w, s, a);
  }
  // Same sum as exact (src/fmma.cpp:103-141 builds the dense matrix first).
  void exact_matvec(const std::vector<point>& t, const std::vector<point>& s, std::vector<TYPE>& a) { run("exact", t, nullptr, s, a); }
  void exact_matvec(const std::vector<point>& t, const std::vector<TYPE>& w, const std::vector<point>& s, std::vector<TYPE>& a) {
    run("exact", t, &w, s, a);
  }
  void fmm(const std::vector<point>& t, const std::vector<point>& s, std::vector<TYPE>& a) { run("fmm", t, nullptr, s, a); }
  void fmm(const std::vector<point>& t, const std::vector<TYPE>& w, const std::vector<point>& s, std::vector<TYPE>& a) {
    run("fmm", t, &w, s, a);
  }
  void tree(const std::vector<point>& t, const std::vector<point>& s, std::vector<TYPE>& a) { run("tree", t, nullptr, s, a); }
  void tree(const std::vector<point>& t, const std::vector<TYPE>& w, const std::vector<point>& s, std::vector<TYPE>& a) {
    run("tree", t, &w, s, a);
  }
  void nrnmm(const std::vector<point>& t, const std::vector<point>& s, std::vector<TYPE>& a) { run("nrnmm", t, nullptr, s, a); }
  void nrnmm(const std::vector<point>& t, const std::vector<TYPE>& w, const std::vector<point>& s, std::vector<TYPE>& a) {
    run("nrnmm", t, &w, s, a);
  }

  const std::map<std::string, double>& get_time_log() const { return time_log; }

 protected:
  // Cube of targets then sources (src/fmm_core.cpp:125-173), on the host.
  void get_origin_and_length(const std::vector<point>& a1, const std::vector<point>& a2, point& origin, TYPE& Len) {
    point mn{}, mx{};
    if (!a1.empty()) mn = mx = a1[0];
    else if (!a2.empty()) mn = mx = a2[0];
    for (const auto* v : {&a1, &a2})
      for (const point& p : *v)
        for (std::size_t d = 0; d < DIM; ++d) {
          mn[d] = std::min(mn[d], p[d]);
          mx[d] = std::max(mx[d], p[d]);
        }
    Len = 0;
    for (std::size_t d = 0; d < DIM; ++d) Len = std::max(Len, (TYPE)(mx[d] - mn[d]));
    for (std::size_t d = 0; d < DIM; ++d) origin[d] = (mx[d] + mn[d]) / 2 - Len / 2;
  }

  std::map<std::string, double> time_log;

 private:
  void host_functor() {
    fail(FMMA_ERR_INVALID_ARG,
         "a host std::function kernel cannot run on the GPU: use fmma::kernels::* or set_fn_device (fmma/device.cuh)");
  }

  [[noreturn]] void fail_exit(const std::string& msg) {
    std::fprintf(stderr, "%s:%d ERROR : %s\n", __FILE__, __LINE__, msg.c_str());
    std::exit(EXIT_FAILURE);
  }
  void fail(int status, const std::string& msg) {
    if (throw_) throw Error(status, msg);
    fail_exit(msg);
  }
  void check(fmma_status st) {
    if (st != FMMA_OK) fail(st, fmma_last_error());
  }

  fmma_ctx* context() {
    if (!ctx_) check(fmma_ctx_create(device_, &ctx_));
    return ctx_;
  }

  void run(const std::string& solver, const std::vector<point>& target, const std::vector<TYPE>* w,
           const std::vector<point>& source, std::vector<TYPE>& ans) {
    const auto start = std::chrono::system_clock::now();
    int sid;
    // exact_matvec forms the dense matrix first (src/fmma.cpp:103-141): the same sum
    if (solver == "exact" || solver == "exact_matvec") sid = FMMA_SOLVER_EXACT;
    else if (solver == "fmm") sid = FMMA_SOLVER_FMM;
    else if (solver == "tree") sid = FMMA_SOLVER_TREE;
    else if (solver == "nrnmm") sid = FMMA_SOLVER_NRNMM;
    else
      return fail(FMMA_ERR_UNSUPPORTED_SOLVER, "solve type " + solver + " not undefined");
    const int64_t nt = (int64_t)target.size(), ns = (int64_t)source.size();
    ans.resize(target.size());
    if (w && (int64_t)w->size() != ns)
      return fail(FMMA_ERR_INVALID_ARG, "source_weight size (" + std::to_string(w->size()) + ") != source size (" +
                                            std::to_string(source.size()) + ")");
    if ((sid == FMMA_SOLVER_FMM || sid == FMMA_SOLVER_TREE) && Depth_ <= 0)
      Depth_ = fmma_default_depth(nt > 0 ? nt : 1, (int)DIM);  // sticky (src/fmm.cpp:23-28, src/tree.cpp:21-26)
    fmma_ctx* c = context();
    if (expr_) {
      // installed on the context by set_fn_expr
    } else if (user_hook_) {
      check(fmma_set_user_kernel(c, user_hook_, user_obj_.get(), user_ti_ ? 1 : 0));
    } else {
      check(fmma_set_kernel(c, kernel_.id, kernel_.p0));
    }
    // nrnmm takes nrn_N in the depth slot; the default it picks sticks, like the
    // reference's member (src/nrnmm.cpp:20-22)
    const int depth = sid == FMMA_SOLVER_NRNMM ? nrn_N_ : Depth_;
    int used = 0;
    const TYPE* tp = nt ? target[0].data() : nullptr;
    const TYPE* sp = ns ? source[0].data() : nullptr;
    const TYPE* wp = w ? w->data() : nullptr;
    fmma_status st;
    if (std::is_same<TYPE, double>::value)
      st = fmma_solve_d(c, (int)DIM, sid, poly_ord_, depth, trans_sym_flag_, precision_, nt, (const double*)tp, ns,
                        (const double*)sp, 1, (const double*)wp, (double*)ans.data(), FMMA_MEM_HOST, &used);
    else
      st = fmma_solve_f(c, (int)DIM, sid, poly_ord_, depth, trans_sym_flag_, precision_, nt, (const float*)tp, ns,
                        (const float*)sp, 1, (const float*)wp, (float*)ans.data(), FMMA_MEM_HOST, &used);
    check(st);
    if (sid == FMMA_SOLVER_NRNMM) nrn_N_ = used;
    double ms[FMMA_NUM_STAGES] = {0};
    fmma_stage_times(c, ms, FMMA_NUM_STAGES);
    for (int i = 1; i < 7; ++i)
      if (ms[i] > 0) time_log[fmma_stage_name(i)] += ms[i];
    const auto end = std::chrono::system_clock::now();
    time_log["total time(" + solver + ")"] =
        (double)std::chrono::duration_cast<std::chrono::milliseconds>(end - start).count();
  }

  std::string solver_type_ = "exact";  // include/fmma/fmma.hpp:90
  int nrn_N_ = -1;
  int poly_ord_ = 1;
  int Depth_ = -1;
  int trans_sym_flag_ = 0;
  int precision_ = FMMA_PREC_FP64;
  int device_ = 0;
  bool throw_ = false;
  kernels::Kernel kernel_ = kernels::inv_r();
  fmma_user_hook user_hook_ = nullptr;
  std::shared_ptr<void> user_obj_;
  bool expr_ = false;
  bool user_ti_ = true;
  fmma_ctx* ctx_ = nullptr;
};

}  // namespace fmma
