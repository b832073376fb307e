// kernels.cuh — built-in interaction kernels f(x, y) as device functions,
// their gradients (adjoint) and compile-time dispatch over (kernel, dim).
//
// The ids and formulas match include/fmma_b200.h and the CPU oracle.  The
// reference's default functor is include/fmma/fmma.hpp:55-63 (1/|x-y|).
#pragma once

#include <cuda_runtime.h>

#include "../../include/fmma_b200.h"

namespace fmma_b200 {

template <int KID>
struct KernelTraits {
  static constexpr bool translation_invariant = KID != FMMA_KERNEL_SUM2_OVER_R2;
  static constexpr bool symmetric = KID != FMMA_KERNEL_INV_DIFF && KID != FMMA_KERNEL_SUM_OVER_R2;
};

inline bool kernel_translation_invariant(int kid) { return kid != FMMA_KERNEL_SUM2_OVER_R2; }

// FP64 evaluation.
template <int KID, int D>
__device__ __forceinline__ double keval(const double* x, const double* y, double p0) {
  double r2 = 0.0, s = 0.0;
  if (KID == FMMA_KERNEL_INV_DIFF) {
    double t = x[0] - y[0];
    return t != 0.0 ? 1.0 / t : 0.0;
  }
#pragma unroll
  for (int q = 0; q < D; ++q) {
    double t = x[q] - y[q];
    r2 += t * t;
    if (KID == FMMA_KERNEL_SUM_OVER_R2) s += t;
    if (KID == FMMA_KERNEL_SUM2_OVER_R2) { double u = x[q] + y[q]; s += u * u; }
  }
  switch (KID) {
    case FMMA_KERNEL_INV_R: return 1.0 / sqrt(r2);
    case FMMA_KERNEL_INV_R_SAFE: return r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0;
    case FMMA_KERNEL_LOG_R: return r2 > 0.0 ? 0.5 * log(r2) : 0.0;
    case FMMA_KERNEL_GAUSSIAN: return exp(-r2 / p0);
    case FMMA_KERNEL_MULTIQUADRIC: return sqrt(r2 + p0);
    case FMMA_KERNEL_SUM_OVER_R2: return s / r2;
    case FMMA_KERNEL_SUM2_OVER_R2: return s / r2;
    default: return 0.0;
  }
}

// FP32 evaluation on a difference vector t = x - y (translation-invariant
// kernels only; the mixed-precision P2P forms t from box-local offsets).
template <int KID, int D>
__device__ __forceinline__ float keval_diff_f32(const float* t, float p0) {
  if (KID == FMMA_KERNEL_INV_DIFF) return t[0] != 0.f ? 1.f / t[0] : 0.f;
  float r2 = 0.f, s = 0.f;
#pragma unroll
  for (int q = 0; q < D; ++q) {
    r2 = fmaf(t[q], t[q], r2);
    if (KID == FMMA_KERNEL_SUM_OVER_R2) s += t[q];
  }
  switch (KID) {
    case FMMA_KERNEL_INV_R: return rsqrtf(r2);
    case FMMA_KERNEL_INV_R_SAFE: return r2 > 0.f ? rsqrtf(r2) : 0.f;
    case FMMA_KERNEL_LOG_R: return r2 > 0.f ? 0.5f * __logf(r2) : 0.f;
    case FMMA_KERNEL_GAUSSIAN: return __expf(-r2 / p0);
    case FMMA_KERNEL_MULTIQUADRIC: return sqrtf(r2 + p0);
    case FMMA_KERNEL_SUM_OVER_R2: return s / r2;
    default: return 0.f;
  }
}

// Gradient of f with respect to its first argument x, FP64 (adjoint).
// grad_y f = -grad_x f for translation-invariant kernels.
template <int KID, int D>
__device__ __forceinline__ void kgrad_x(const double* x, const double* y, double p0, double* g) {
  double t[D];
  double r2 = 0.0, s = 0.0;
#pragma unroll
  for (int q = 0; q < D; ++q) {
    t[q] = x[q] - y[q];
    r2 += t[q] * t[q];
    s += t[q];
  }
  double c = 0.0;
  switch (KID) {
    case FMMA_KERNEL_INV_R:
    case FMMA_KERNEL_INV_R_SAFE: {
      if (r2 > 0.0) { double ir = 1.0 / sqrt(r2); c = -ir * ir * ir; }
      break;
    }
    case FMMA_KERNEL_LOG_R: c = r2 > 0.0 ? 1.0 / r2 : 0.0; break;
    case FMMA_KERNEL_GAUSSIAN: c = -2.0 / p0 * exp(-r2 / p0); break;
    case FMMA_KERNEL_MULTIQUADRIC: c = 1.0 / sqrt(r2 + p0); break;
    case FMMA_KERNEL_INV_DIFF: {
      g[0] = t[0] != 0.0 ? -1.0 / (t[0] * t[0]) : 0.0;
      return;
    }
    case FMMA_KERNEL_SUM_OVER_R2: {
#pragma unroll
      for (int q = 0; q < D; ++q) g[q] = r2 > 0.0 ? (1.0 / r2 - 2.0 * s * t[q] / (r2 * r2)) : 0.0;
      return;
    }
    default: {
#pragma unroll
      for (int q = 0; q < D; ++q) g[q] = 0.0;
      return;
    }
  }
#pragma unroll
  for (int q = 0; q < D; ++q) g[q] = c * t[q];
}

// Host dispatch helper: calls F::template run<KID, D>(args...).
template <typename F, typename... Args>
void dispatch_kernel(int kid, int dim, Args&&... args) {
#define FMMA_DISPATCH_D(KID_)                                          \
  switch (dim) {                                                        \
    case 1: F::template run<KID_, 1>(args...); return;                  \
    case 2: F::template run<KID_, 2>(args...); return;                  \
    default: F::template run<KID_, 3>(args...); return;                 \
  }
  switch (kid) {
    case FMMA_KERNEL_INV_R: FMMA_DISPATCH_D(FMMA_KERNEL_INV_R)
    case FMMA_KERNEL_INV_R_SAFE: FMMA_DISPATCH_D(FMMA_KERNEL_INV_R_SAFE)
    case FMMA_KERNEL_INV_DIFF: F::template run<FMMA_KERNEL_INV_DIFF, 1>(args...); return;
    case FMMA_KERNEL_LOG_R: FMMA_DISPATCH_D(FMMA_KERNEL_LOG_R)
    case FMMA_KERNEL_GAUSSIAN: FMMA_DISPATCH_D(FMMA_KERNEL_GAUSSIAN)
    case FMMA_KERNEL_MULTIQUADRIC: FMMA_DISPATCH_D(FMMA_KERNEL_MULTIQUADRIC)
    case FMMA_KERNEL_SUM_OVER_R2: FMMA_DISPATCH_D(FMMA_KERNEL_SUM_OVER_R2)
    default: FMMA_DISPATCH_D(FMMA_KERNEL_SUM2_OVER_R2)
  }
#undef FMMA_DISPATCH_D
}

}  // namespace fmma_b200
