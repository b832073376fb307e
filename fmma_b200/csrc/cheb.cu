// cheb.cu — global Chebyshev approximation on [-1, 1]^dim
// (src/chebyshev_approx.cpp:36-97, include/fmma/chebyshev_approx.hpp).
//
// f(x) ~ sum_i coef[i] prod_q T_{i_q}(x_q), i_q in [0, nth], flat index
// i = sum_q i_q (nth + 1)^q (dimension 0 fastest, as the reference orders
// both its nodes and its coefficients).
//
// Fit: the reference builds the (nth+1)^dim square system
// Mat[i][j] = prod_q T_{j_q}(x_{i_q}) at the tensor Chebyshev nodes
// x_k = cos((2k + 1) pi / (2 (nth + 1))) and solves Mat coef = f(nodes) by
// GCR from a random start (src/math.cpp:371-440, stopping at a squared
// residual of 1e-6).  Mat is the tensor power of the 1-D matrix
// C[k][j] = T_j(x_k), whose columns are orthogonal at these nodes
// (C^T C = diag(n, n/2, .., n/2), n = nth + 1), so the exact solution is
// coef = (A (x) .. (x) A) f with A = diag(1/n, 2/n, ..) C^T: one pass of a
// 1-D transform per dimension, applied here to many functions at once.
//
// Evaluation: four points per thread, the innermost dimension summed by
// Clenshaw's recurrence and the outer ones by the three-term recurrence of
// T_k; each coefficient is one warp-uniform load shared by the thread's four
// points (2 FP64 operations per coefficient and point: FP64-pipe bound).
// The reference rejects points outside [-1, 1] (Chebyshev,
// src/math.cpp:14-26); here such a point is reported as
// FMMA_ERR_INVALID_ARG after the launch.
#include <cmath>
#include <vector>

#include "fmma_internal.cuh"

namespace fmma_b200 {

namespace {

// out[f][.., j at dimension q, ..] = sum_k A[j][k] in[f][.., k, ..]
__global__ void k_cheb_pass(const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ A,
                            int n, int64_t stride, int64_t total) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)((e / stride) % n);
    const int64_t base = e - (int64_t)j * stride;
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += A[j * n + k] * in[base + (int64_t)k * stride];
    out[e] = s;
  }
}

// s[j] = sum_{k < n} c[k] T_k(x[j]) for PPT points by Clenshaw's recurrence,
// one coefficient load shared by the PPT points.
template <int PPT>
__device__ __forceinline__ void clenshaw(const double* __restrict__ c, int n, const double* x, double* s) {
  double b1[PPT], b2[PPT];
#pragma unroll
  for (int j = 0; j < PPT; ++j) b1[j] = b2[j] = 0.0;
  for (int k = n - 1; k >= 1; --k) {
    const double ck = __ldg(c + k);
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const double b0 = fma(2.0 * x[j], b1[j], ck - b2[j]);
      b2[j] = b1[j];
      b1[j] = b0;
    }
  }
  const double c0 = __ldg(c);
#pragma unroll
  for (int j = 0; j < PPT; ++j) s[j] = fma(x[j], b1[j], c0 - b2[j]);
}

// acc[j] += T_i(x[j]) * s[j] over i by the three-term recurrence: the
// recurrence state (t0 = T_{i-1}, t1 = T_i) advances after each use.
template <int PPT>
struct ChebWalk {
  double t0[PPT], t1[PPT];
  __device__ __forceinline__ void start() {
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      t0[j] = 0.0;
      t1[j] = 1.0;
    }
  }
  __device__ __forceinline__ void step(const double* x, int i) {
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const double t2 = i == 0 ? x[j] : 2.0 * x[j] * t1[j] - t0[j];
      t0[j] = t1[j];
      t1[j] = t2;
    }
  }
};

// PPT points per thread: point base + j * blockDim + thread for j < PPT.
template <int D, int PPT>
__global__ void __launch_bounds__(256) k_cheb_eval(const double* __restrict__ coef, int n, int64_t size, int nfunc,
                                                   const double* __restrict__ pts, int64_t npts,
                                                   double* __restrict__ out, int* __restrict__ bad) {
  const int64_t span = (int64_t)blockDim.x * PPT;
  for (int64_t base = (int64_t)blockIdx.x * span; base < npts; base += (int64_t)gridDim.x * span) {
    double x[D][PPT];
    bool in[PPT], ok[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const int64_t p = base + (int64_t)j * blockDim.x + threadIdx.x;
      in[j] = p < npts;
      ok[j] = true;
#pragma unroll
      for (int q = 0; q < D; ++q) {
        x[q][j] = in[j] ? pts[p * D + q] : 0.0;
        ok[j] = ok[j] && x[q][j] >= -1.0 && x[q][j] <= 1.0;  // false for NaN as well
      }
      if (in[j] && !ok[j]) atomicOr(bad, 1);
    }
    for (int f = 0; f < nfunc; ++f) {
      const double* c = coef + (int64_t)f * size;
      double acc[PPT];
      if constexpr (D == 1) {
        clenshaw<PPT>(c, n, x[0], acc);
      } else if constexpr (D == 2) {
#pragma unroll
        for (int j = 0; j < PPT; ++j) acc[j] = 0.0;
        ChebWalk<PPT> w1;
        w1.start();
        for (int i1 = 0; i1 < n; ++i1) {
          double s[PPT];
          clenshaw<PPT>(c + (int64_t)i1 * n, n, x[0], s);
#pragma unroll
          for (int j = 0; j < PPT; ++j) acc[j] = fma(w1.t1[j], s[j], acc[j]);
          w1.step(x[1], i1);
        }
      } else {
#pragma unroll
        for (int j = 0; j < PPT; ++j) acc[j] = 0.0;
        ChebWalk<PPT> w2;
        w2.start();
        for (int i2 = 0; i2 < n; ++i2) {
          double m[PPT];
#pragma unroll
          for (int j = 0; j < PPT; ++j) m[j] = 0.0;
          ChebWalk<PPT> w1;
          w1.start();
          for (int i1 = 0; i1 < n; ++i1) {
            double s[PPT];
            clenshaw<PPT>(c + ((int64_t)i2 * n + i1) * n, n, x[0], s);
#pragma unroll
            for (int j = 0; j < PPT; ++j) m[j] = fma(w1.t1[j], s[j], m[j]);
            w1.step(x[1], i1);
          }
#pragma unroll
          for (int j = 0; j < PPT; ++j) acc[j] = fma(w2.t1[j], m[j], acc[j]);
          w2.step(x[2], i2);
        }
      }
#pragma unroll
      for (int j = 0; j < PPT; ++j) {
        const int64_t p = base + (int64_t)j * blockDim.x + threadIdx.x;
        if (in[j]) out[(int64_t)f * npts + p] = ok[j] ? acc[j] : nan("");
      }
    }
  }
}

// A[j][k] = (j == 0 ? 1 : 2) / n * T_j(x_k), T_j(x_k) = cos(j (2k + 1) pi / (2n)).
std::vector<double> fit_matrix(int n) {
  std::vector<double> A((size_t)n * n);
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k)
      A[(size_t)j * n + k] = (j == 0 ? 1.0 : 2.0) / n * std::cos(j * (2.0 * k + 1.0) / (2.0 * n) * M_PI);
  return A;
}

}  // namespace

void cheb_fit(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* values, double* coef) {
  const int n = nth + 1;
  int64_t size = 1;
  for (int q = 0; q < dim; ++q) size *= n;
  const int64_t total = size * nfunc;
  const std::vector<double> A = fit_matrix(n);
  double* dA = ctx_buf_t<double>(ctx, "cheb_fit_A", A.size());
  upload(ctx, dA, A.data(), sizeof(double) * A.size());
  // ping-pong: pass q reads src, writes dst; the last pass lands in coef
  double* tmp = ctx_buf_t<double>(ctx, "cheb_fit_tmp", (size_t)total);
  const double* src = values;
  int64_t stride = 1;
  for (int q = 0; q < dim; ++q) {
    double* dst = ((dim - 1 - q) % 2 == 0) ? coef : tmp;
    FMMA_LAUNCH(ctx, k_cheb_pass, grid_for(total, 256), 256, 0, src, dst, dA, n, stride, total);
    src = dst;
    stride *= n;
  }
}

void cheb_eval(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* coef, int64_t npts, const double* pts,
               double* out) {
  const int n = nth + 1;
  int64_t size = 1;
  for (int q = 0; q < dim; ++q) size *= n;
  int* bad = ctx_buf_t<int>(ctx, "cheb_bad", 1);
  FMMA_CHECK_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
  constexpr int kPPT = 4;
  const unsigned g = grid_for((npts + kPPT - 1) / kPPT, 256, (int64_t)ctx->sm_count * 8);
  if (dim == 1) FMMA_LAUNCH(ctx, (k_cheb_eval<1, kPPT>), g, 256, 0, coef, n, size, nfunc, pts, npts, out, bad);
  else if (dim == 2) FMMA_LAUNCH(ctx, (k_cheb_eval<2, kPPT>), g, 256, 0, coef, n, size, nfunc, pts, npts, out, bad);
  else FMMA_LAUNCH(ctx, (k_cheb_eval<3, kPPT>), g, 256, 0, coef, n, size, nfunc, pts, npts, out, bad);
  int h = 0;
  read_ints(ctx, bad, &h, 1);
  if (h) throw Error(FMMA_ERR_INVALID_ARG, "Chebyshev evaluation point outside [-1, 1] (or NaN)");
}

}  // namespace fmma_b200
