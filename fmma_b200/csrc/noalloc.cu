// noalloc.cu — fmma_exact_noalloc_d: the exact direct sum for small target
// sets that allocates nothing.
//
// A variant of the exact kernel (src/fmma.cpp:80-94) that splits the source
// range over the blocks of a second grid dimension, so that a few hundred or
// thousand targets still fill all SMs.  Each (target tile, source chunk)
// block writes its partial sums to scratch; a second kernel adds the chunks
// in a fixed order, so the result does not depend on scheduling.
//
// The scratch is a file-scope device array of kNoAllocScratchBytes (16 MiB),
// not memory from cudaMalloc: the entry point calls no allocator of any kind
// on its success path.  Its device address is looked up on every call, with
// the caller's device current (cudaGetSymbolAddress allocates nothing), so a
// context that was torn down and re-created (cudaDeviceReset) gets the
// array's new address.  The first call on a device also loads every kernel
// instantiation of this file and reads the device's SM count.  Every partial
// sum is written before it is read, so nothing in the scratch needs clearing;
// with no sources the entry point clears `ans` itself.
#include <algorithm>
#include <mutex>

#include "fmma_internal.cuh"
#include "kernels.cuh"

namespace fmma_b200 {

constexpr int kNaThreads = 256;
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr int64_t kNoAllocScratchDoubles = (int64_t)(kNoAllocScratchBytes / sizeof(double));
// nt * nrhs above this cannot be split at least 8 ways inside the scratch
constexpr int64_t kNoAllocMaxOutputs = kNoAllocScratchDoubles / 8;
constexpr int kNaMaxDevices = 64;
constexpr int kNaBlocksPerSm = 8;  // split blocks aimed at per SM

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// part[(s * R + r) * nt + i] = sum over the sources of chunk s (or ans when
// the grid has one chunk).
template <int KID, int D>
__global__ void __launch_bounds__(kNaThreads) k_exact_split(const double* __restrict__ tgt, int64_t nt,
                                                            const double* __restrict__ src, int64_t ns,
                                                            const double* __restrict__ w, int R, double p0,
                                                            int64_t chunk, double* __restrict__ part) {
  __shared__ double sy[kNaThreads][D];
  __shared__ double sw[kNaThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < nt;
  const int64_t j_begin = (int64_t)blockIdx.y * chunk;
  const int64_t j_end = min(ns, j_begin + chunk);
  double x[D];
#pragma unroll
  for (int q = 0; q < D; ++q) x[q] = ok ? tgt[i * D + q] : 0.0;
  for (int r = 0; r < R; ++r) {
    double acc = 0.0;
    for (int64_t j0 = j_begin; j0 < j_end; j0 += kNaThreads) {
      const int cnt = (int)min((int64_t)kNaThreads, j_end - j0);
      __syncthreads();
      if ((int)threadIdx.x < cnt) {
#pragma unroll
        for (int q = 0; q < D; ++q) sy[threadIdx.x][q] = src[(j0 + threadIdx.x) * D + q];
        sw[threadIdx.x] = w ? w[(int64_t)r * ns + j0 + threadIdx.x] : 1.0;
      }
      __syncthreads();
      if (ok)
        for (int j = 0; j < cnt; ++j) acc += sw[j] * keval<KID, D>(x, sy[j], p0);
    }
    if (ok) part[((int64_t)blockIdx.y * R + r) * nt + i] = acc;
  }
}

// ans[e] = sum_{s < S} part[s * nout + e], s ascending.
__global__ void k_exact_split_reduce(const double* __restrict__ part, int S, int64_t nout, double* __restrict__ ans) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nout; e += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += part[(int64_t)s * nout + e];
    ans[e] = acc;
  }
}

namespace {

struct SplitLaunch {
  template <int KID, int D>
  static void run(cudaError_t* err, dim3 grid, cudaStream_t st, const double* tgt, int64_t nt, const double* src,
                  int64_t ns, const double* w, int R, double p0, int64_t chunk, double* part) {
    k_exact_split<KID, D><<<grid, kNaThreads, 0, st>>>(tgt, nt, src, ns, w, R, p0, chunk, part);
    *err = cudaGetLastError();
  }
};

struct LoadAll {
  template <int KID, int D>
  static void run(cudaError_t* err) {
    cudaFuncAttributes a;
    if (*err == cudaSuccess) *err = cudaFuncGetAttributes(&a, k_exact_split<KID, D>);
  }
};

std::mutex g_na_mu;
int g_na_sms[kNaMaxDevices] = {};  // SM count per device, 0 until set up

// Once per device: every kernel of this file loaded (module loading is
// otherwise lazy, at the first launch) and the SM count read.  On every call:
// the scratch's device address in the current context.
cudaError_t na_setup(int dev, double** out, int* sms) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  cudaError_t e = cudaSuccess;
  if (g_na_sms[dev] == 0) {
    for (int kid = 0; kid < FMMA_KERNEL_COUNT && e == cudaSuccess; ++kid)
      for (int dim = 1; dim <= 3 && e == cudaSuccess; ++dim) dispatch_kernel<LoadAll>(kid, dim, &e);
    if (e == cudaSuccess) {
      cudaFuncAttributes a;
      e = cudaFuncGetAttributes(&a, k_exact_split_reduce);
    }
    int n = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_na_sms[dev] = n > 0 ? n : 1;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<double*>(p);
  *sms = g_na_sms[dev];
  return cudaSuccess;
}

fmma_status na_fail(fmma_status code, const char* what) {
  set_last_error(std::string("fmma_exact_noalloc_d: ") + what);
  return code;
}

fmma_status na_cuda_fail(const char* what, cudaError_t e) {
  set_last_error(std::string("fmma_exact_noalloc_d: ") + what + ": " + cudaGetErrorString(e));
  return FMMA_ERR_CUDA;
}

}  // namespace
}  // namespace fmma_b200

using namespace fmma_b200;

extern "C" fmma_status fmma_exact_noalloc_d(int dim, int kernel_id, double p0, int64_t n_tgt, const double* tgt,
                                            int64_t n_src, const double* src, int nrhs, const double* w, double* ans,
                                            void* stream) {
  try {
    if (dim < 1 || dim > 3) return na_fail(FMMA_ERR_INVALID_ARG, "dim must be 1, 2 or 3");
    if (kernel_id < 0 || kernel_id >= FMMA_KERNEL_COUNT) return na_fail(FMMA_ERR_INVALID_ARG, "unknown kernel id");
    if (kernel_id == FMMA_KERNEL_INV_DIFF && dim != 1)
      return na_fail(FMMA_ERR_INVALID_ARG, "kernel 1/(x-y) is one-dimensional");
    if (kernel_id == FMMA_KERNEL_GAUSSIAN && !(p0 > 0.0))
      return na_fail(FMMA_ERR_INVALID_ARG, "Gaussian width p0 must be > 0");
    if (kernel_id == FMMA_KERNEL_MULTIQUADRIC && !(p0 >= 0.0))
      return na_fail(FMMA_ERR_INVALID_ARG, "multiquadric shift p0 must be >= 0");
    if (n_tgt < 0 || n_src < 0) return na_fail(FMMA_ERR_INVALID_ARG, "negative point count");
    if (nrhs < 1 || nrhs > 64) return na_fail(FMMA_ERR_INVALID_ARG, "nrhs must be in [1, 64]");
    if (n_tgt > kNoAllocMaxOutputs || n_tgt * nrhs > kNoAllocMaxOutputs)
      return na_fail(FMMA_ERR_INVALID_ARG,
                     ("n_tgt * nrhs = " + std::to_string(n_tgt) + " * " + std::to_string(nrhs) +
                      " exceeds the limit of " +
                      std::to_string(kNoAllocMaxOutputs) +
                      " set by its 16 MiB static scratch; use fmma_solve_d for larger target sets")
                         .c_str());
    if (n_src >= ((int64_t)1 << 31)) return na_fail(FMMA_ERR_INVALID_ARG, "n_src must be below 2^31");
    if (n_tgt > 0 && (tgt == nullptr || ans == nullptr)) return na_fail(FMMA_ERR_INVALID_ARG, "null pointer");
    if (n_src > 0 && src == nullptr) return na_fail(FMMA_ERR_INVALID_ARG, "null source pointer");
    if (n_tgt == 0) return FMMA_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_cuda_fail("cudaGetDevice", e);
    if (dev < 0 || dev >= kNaMaxDevices) return na_fail(FMMA_ERR_NO_DEVICE, "device index beyond 63");
    double* scratch = nullptr;
    int sms = 0;
    e = na_setup(dev, &scratch, &sms);
    if (e != cudaSuccess) return na_cuda_fail("set-up", e);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nout = n_tgt * nrhs;
    if (n_src == 0) {
      e = cudaMemsetAsync(ans, 0, sizeof(double) * (size_t)nout, st);
      return e == cudaSuccess ? FMMA_OK : na_cuda_fail("cudaMemsetAsync", e);
    }
    // chunks: enough blocks for all SMs, at least kNaThreads sources each,
    // as many partial sums as the scratch holds
    const int64_t tiles = (n_tgt + kNaThreads - 1) / kNaThreads;
    int64_t S = ((int64_t)sms * kNaBlocksPerSm + tiles - 1) / tiles;
    S = std::min(S, (n_src + kNaThreads - 1) / kNaThreads);
    S = std::min(S, kNoAllocScratchDoubles / nout);
    S = std::max<int64_t>(S, 1);
    const int64_t chunk = (n_src + S - 1) / S;
    S = (n_src + chunk - 1) / chunk;
    double* part = S == 1 ? ans : scratch;
    dispatch_kernel<SplitLaunch>(kernel_id, dim, &e, dim3((unsigned)tiles, (unsigned)S), st, tgt, n_tgt, src, n_src, w,
                                 nrhs, p0, chunk, part);
    if (e != cudaSuccess) return na_cuda_fail("k_exact_split launch", e);
    if (S > 1) {
      const int64_t g = std::min<int64_t>((nout + 255) / 256, (int64_t)sms * 16);
      k_exact_split_reduce<<<(unsigned)g, 256, 0, st>>>(scratch, (int)S, nout, ans);
      e = cudaGetLastError();
      if (e != cudaSuccess) return na_cuda_fail("k_exact_split_reduce launch", e);
    }
    return FMMA_OK;
  } catch (const std::exception& ex) {
    set_last_error(ex.what());
    return FMMA_ERR_CUDA;
  }
}
