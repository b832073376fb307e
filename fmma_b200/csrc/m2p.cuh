// m2p.cuh — the inner loop shared by the far-field sums of the tree and
// nrnmm solvers (M2P: a target against the P Chebyshev nodes of a box,
// weighted by the box's expansion; src/fmm_core.cpp:624-661,
// src/nrnmm.cpp:86-97).
//
// A box is staged in shared memory as its 1-D node coordinates X[q][o]
// (D x n) and its weights W[r][k] (RB x P); node k = (o_0, .., o_{D-1}) with
// the last dimension fastest.  The innermost loop is unrolled so that the
// evaluations of consecutive nodes (each a chain of a square root or
// logarithm and a divide) overlap in the FP64 pipe.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace fmma_b200 {

// Kernel value for the far sums: 1/r through rsqrt (one rounding instead of
// the square root and divide of keval, which keeps the near field and exact
// sums bit-comparable with the reference); every other kernel as keval.
template <int KID, int D>
__device__ __forceinline__ double kfar(const double* x, const double* y, double p0) {
  if constexpr (KID == FMMA_KERNEL_INV_R || KID == FMMA_KERNEL_INV_R_SAFE) {
    double r2 = 0.0;
#pragma unroll
    for (int q = 0; q < D; ++q) {
      const double t = x[q] - y[q];
      r2 += t * t;
    }
    if constexpr (KID == FMMA_KERNEL_INV_R_SAFE) return r2 > 0.0 ? rsqrt(r2) : 0.0;
    return rsqrt(r2);
  } else {
    return keval<KID, D>(x, y, p0);
  }
}

template <int KID, int D, int RB>
__device__ __forceinline__ void far_box_sum(const double* x, const double* __restrict__ X,
                                            const double* __restrict__ W, int n, int P, double p0, double* acc) {
  double y[D];
  if constexpr (D == 1) {
#pragma unroll 4
    for (int o0 = 0; o0 < n; ++o0) {
      y[0] = X[o0];
      const double f = kfar<KID, D>(x, y, p0);
#pragma unroll
      for (int rr = 0; rr < RB; ++rr) acc[rr] += f * W[rr * P + o0];
    }
  } else if constexpr (D == 2) {
    for (int o0 = 0; o0 < n; ++o0) {
      y[0] = X[o0];
      const double* Wk = W + o0 * n;
#pragma unroll 4
      for (int o1 = 0; o1 < n; ++o1) {
        y[1] = X[n + o1];
        const double f = kfar<KID, D>(x, y, p0);
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) acc[rr] += f * Wk[rr * P + o1];
      }
    }
  } else {
    for (int o0 = 0; o0 < n; ++o0) {
      y[0] = X[o0];
      for (int o1 = 0; o1 < n; ++o1) {
        y[1] = X[n + o1];
        const double* Wk = W + (o0 * n + o1) * n;
#pragma unroll 4
        for (int o2 = 0; o2 < n; ++o2) {
          y[2] = X[2 * n + o2];
          const double f = kfar<KID, D>(x, y, p0);
#pragma unroll
          for (int rr = 0; rr < RB; ++rr) acc[rr] += f * Wk[rr * P + o2];
        }
      }
    }
  }
}

}  // namespace fmma_b200
