// fmm_stages.cuh — device helpers shared by the FMM stage kernels.
#pragma once

#include <cuda_runtime.h>

#include "fmma_internal.cuh"

namespace fmma_b200 {

// Leaf coordinate of one point along one dimension (src/fmm_core.cpp:261):
// min((int)((x - origin) / (Len / N)), N - 1), in the caller's precision.
template <typename T>
__device__ __forceinline__ int bin_coord(T x, const Cube& c, int q, int N);
template <>
__device__ __forceinline__ int bin_coord<double>(double x, const Cube& c, int q, int N) {
  double len = __ddiv_rn(c.Len, (double)N);
  int t = __double2int_rz(__ddiv_rn(__dsub_rn(x, c.origin[q]), len));
  return t < N - 1 ? t : N - 1;
}
template <>
__device__ __forceinline__ int bin_coord<float>(float x, const Cube& c, int q, int N) {
  float len = __fdiv_rn(c.Lenf, (float)N);
  int t = __float2int_rz(__fdiv_rn(__fsub_rn(x, c.originf[q]), len));
  return t < N - 1 ? t : N - 1;
}

// Local coordinate of a point in its leaf, in [-1, 1] (src/fmm_core.cpp:261-264
// and :595-596), in the caller's coordinate precision.  For float inputs the
// reference computes (x-o)/len in float and the affine map in double, then
// stores a float; the same steps are taken here.
__device__ __forceinline__ double point_rel(double x, const Cube& c, int q, int N, bool isf) {
  if (!isf) {
    double len = __ddiv_rn(c.Len, (double)N);
    double qq = __ddiv_rn(__dsub_rn(x, c.origin[q]), len);
    int t = __double2int_rz(qq);
    t = t < N - 1 ? t : N - 1;
    double r = __dsub_rn(__dmul_rn(2.0, __dsub_rn(qq, (double)t)), 1.0);
    r = r < 1.0 ? r : 1.0;
    r = r > -1.0 ? r : -1.0;
    return r;
  }
  float xf = (float)x;
  float len = __fdiv_rn(c.Lenf, (float)N);
  float qq = __fdiv_rn(__fsub_rn(xf, c.originf[q]), len);
  int t = __float2int_rz(qq);
  t = t < N - 1 ? t : N - 1;
  double r = __dsub_rn(__dmul_rn(2.0, (double)__fsub_rn(qq, (float)t)), 1.0);
  r = r < 1.0 ? r : 1.0;
  r = r > -1.0 ? r : -1.0;
  return (double)(float)r;
}

// S_n(node_k, y) for k = 0..n-1 (src/math.cpp:32-50):
// 1/n + 2/n sum_{j=1}^{n-1} T_j(node_k) T_j(y), with T_j(y) by the
// three-term recurrence and T_j(node_k) from the table Tn[k*n + j].
__device__ __forceinline__ void cheb_factors(double y, int n, const double* Tn, double* out) {
  double Tj[kMaxNodes];
  Tj[0] = 1.0;
  if (n > 1) Tj[1] = y;
  for (int j = 2; j < n; ++j) Tj[j] = 2.0 * y * Tj[j - 1] - Tj[j - 2];
  const double inv = 1.0 / n;
  for (int k = 0; k < n; ++k) {
    double s = 0.0;
    for (int j = 1; j < n; ++j) s += Tn[k * n + j] * Tj[j];
    out[k] = inv + 2.0 * inv * s;
  }
}

// S_n(node_k, y) and dS_n/dy for k = 0..n-1: T_j'(y) = j U_{j-1}(y) with the
// second-kind recurrence U_0 = 1, U_1 = 2y, U_{j+1} = 2y U_j - U_{j-1}.
__device__ __forceinline__ void cheb_factors_grad(double y, int n, const double* Tn, double* out, double* dout) {
  double Tj[kMaxNodes], Uj[kMaxNodes];
  Tj[0] = 1.0;
  Uj[0] = 1.0;
  if (n > 1) { Tj[1] = y; Uj[1] = 2.0 * y; }
  for (int j = 2; j < n; ++j) {
    Tj[j] = 2.0 * y * Tj[j - 1] - Tj[j - 2];
    Uj[j] = 2.0 * y * Uj[j - 1] - Uj[j - 2];
  }
  const double inv = 1.0 / n;
  for (int k = 0; k < n; ++k) {
    double s = 0.0, ds = 0.0;
    for (int j = 1; j < n; ++j) {
      s += Tn[k * n + j] * Tj[j];
      ds += Tn[k * n + j] * (double)j * Uj[j - 1];
    }
    out[k] = inv + 2.0 * inv * s;
    dout[k] = 2.0 * inv * ds;
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

}  // namespace fmma_b200
