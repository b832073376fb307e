// prims.cu — device-wide scan and stable LSD radix sort (hand-written), plus
// the context's scratch management and stage timing.
#include <algorithm>
#include <cstring>

#include "fmma_internal.cuh"

namespace fmma_b200 {

// ---------------------------------------------------------------------------
// scratch
// ---------------------------------------------------------------------------
void* dev_alloc(fmma_ctx* ctx, size_t bytes) {
  if (ctx->alloc_fn) {
    void* p = ctx->alloc_fn(bytes, (void*)ctx->stream, ctx->alloc_user);
    if (p && ((uintptr_t)p & 255u) != 0) {  // vector loads and TMA need aligned bases
      if (ctx->free_fn) ctx->free_fn(p, bytes, (void*)ctx->stream, ctx->alloc_user);  // never used
      throw Error(FMMA_ERR_INVALID_ARG, "the context's allocator returned a block not aligned to 256 bytes");
    }
    return p;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void dev_free(fmma_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  if (ctx->alloc_fn) {
    if (ctx->free_fn) ctx->free_fn(p, bytes, (void*)ctx->stream, ctx->alloc_user);
  } else {
    cudaFree(p);
  }
}

void release_device_memory(fmma_ctx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->bufs) dev_free(ctx, kv.second.p, kv.second.bytes);
  for (auto& kv : ctx->ops) dev_free(ctx, kv.second.p, kv.second.bytes);
  ctx->bufs.clear();
  ctx->ops.clear();
}

void* ctx_buf(fmma_ctx* ctx, const std::string& name, size_t bytes) {
  DevBuf& b = ctx->bufs[name];
  if (b.bytes < bytes) {
    if (b.p) {
      FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
      dev_free(ctx, b.p, b.bytes);
      b.p = nullptr;
      b.bytes = 0;
    }
    size_t want = bytes + bytes / 8 + 256;
    b.p = dev_alloc(ctx, want);
    if (!b.p)
      throw Error(FMMA_ERR_OOM, "device allocation of " + std::to_string(want) + " bytes for '" + name +
                                    "' failed");
    b.bytes = want;
  }
  return b.p;
}

void* ctx_pinned(fmma_ctx* ctx, size_t bytes) {
  if (ctx->pinned_bytes < bytes) {
    if (ctx->pinned) {
      FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
      FMMA_CHECK_CUDA(cudaFreeHost(ctx->pinned));
    }
    size_t want = bytes < 4096 ? 4096 : bytes;
    FMMA_CHECK_CUDA(cudaMallocHost(&ctx->pinned, want));
    ctx->pinned_bytes = want;
  }
  return ctx->pinned;
}

void upload(fmma_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (ctx->capturing || bytes == 0) return;
  if (ctx->up_used + bytes > ctx->up_cap) {
    // arena full: wait for the copies in flight from it, then start over
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->up_used = 0;
    if (bytes > ctx->up_cap) {
      if (ctx->up_host) FMMA_CHECK_CUDA(cudaFreeHost(ctx->up_host));
      ctx->up_host = nullptr;
      ctx->up_cap = 0;
      const size_t want = std::max(bytes, (size_t)4 << 20);
      FMMA_CHECK_CUDA(cudaMallocHost((void**)&ctx->up_host, want));
      ctx->up_cap = want;
    }
  }
  char* h = ctx->up_host + ctx->up_used;
  std::memcpy(h, src, bytes);
  ctx->up_used += (bytes + 255) & ~(size_t)255;
  FMMA_CHECK_CUDA(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
}

// The bounded-wait error flags of the tensor-core M2L, one slot per virtual
// level in one small buffer, so the host reads all of them with one copy.
constexpr int kErrSlots = 64;

int* m2l_err_slot(fmma_ctx* ctx, int v) {
  FMMA_REQUIRE(v >= 0 && v < kErrSlots, "too many levels");
  return ctx_buf_t<int>(ctx, "tc_err_all", kErrSlots) + v;
}

void check_m2l_errs(fmma_ctx* ctx, const std::vector<int*>& flags) {
  if (flags.empty()) return;
  const int* base = ctx_buf_t<int>(ctx, "tc_err_all", kErrSlots);
  int h[kErrSlots];
  FMMA_CHECK_CUDA(cudaMemcpy(h, base, sizeof(h), cudaMemcpyDeviceToHost));
  for (const int* f : flags)
    if (h[f - base]) throw Error(FMMA_ERR_TIMEOUT, "tensor-core M2L: a bounded pipeline wait gave up");
}

void read_ints(fmma_ctx* ctx, const int* dev, int* host, int n) {
  int* p = static_cast<int*>(ctx_pinned(ctx, sizeof(int) * (size_t)n));
  FMMA_CHECK_CUDA(cudaMemcpyAsync(p, dev, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(host, p, sizeof(int) * (size_t)n);
}

// ---------------------------------------------------------------------------
// stage timing
// ---------------------------------------------------------------------------
void stages_reset(fmma_ctx* ctx) {
  for (int i = 0; i < FMMA_NUM_STAGES; ++i) {
    ctx->ev_used[i] = false;
    ctx->stage_ms[i] = 0.0;
  }
  ctx->launches = 0;
  ctx->ktimed = 0;
  ctx->m2l_kernel_ms = 0.0;
  ctx->m2l_flops = 0.0;
  ctx->m2l_launches = 0;
  ctx->m2l_err_flags.clear();
}

void kernel_timer_begin(fmma_ctx* ctx) {
  if (ctx->capturing || ctx->ktimed >= fmma_ctx::kMaxTimed) return;
  int i = ctx->ktimed;
  if (!ctx->kev[2 * i]) {
    FMMA_CHECK_CUDA(cudaEventCreate(&ctx->kev[2 * i]));
    FMMA_CHECK_CUDA(cudaEventCreate(&ctx->kev[2 * i + 1]));
  }
  FMMA_CHECK_CUDA(cudaEventRecord(ctx->kev[2 * i], ctx->stream));
}

void kernel_timer_end(fmma_ctx* ctx, double flops_per_pair, int tag) {
  ctx->m2l_launches++;
  if (ctx->capturing || ctx->ktimed >= fmma_ctx::kMaxTimed) return;
  int i = ctx->ktimed++;
  FMMA_CHECK_CUDA(cudaEventRecord(ctx->kev[2 * i + 1], ctx->stream));
  ctx->kflops[i] = flops_per_pair;
  ctx->ktag[i] = tag;
}

void stage_begin(fmma_ctx* ctx, Stage s) {
  if (ctx->capturing) return;
  FMMA_CHECK_CUDA(cudaEventRecord(ctx->ev[2 * s], ctx->stream));
}

void stage_end(fmma_ctx* ctx, Stage s) {
  if (ctx->capturing) return;
  FMMA_CHECK_CUDA(cudaEventRecord(ctx->ev[2 * s + 1], ctx->stream));
  ctx->ev_used[s] = true;
}

void stages_collect(fmma_ctx* ctx) {
  FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  tree_read_pairs(ctx);  // no wait of its own once the stream is idle
  for (int i = 0; i < ctx->ktimed; ++i) {
    float ms = 0.f;
    FMMA_CHECK_CUDA(cudaEventElapsedTime(&ms, ctx->kev[2 * i], ctx->kev[2 * i + 1]));
    ctx->kms[i] = ms;
    ctx->m2l_kernel_ms += ms;
    const int v = ctx->ktag[i];
    if (v >= 0 && v < (int)ctx->tree.lev.size()) {
      ctx->kflops[i] *= (double)ctx->tree.lev[(size_t)v].il_pairs;
      ctx->m2l_flops += ctx->kflops[i];
    }
  }
  check_m2l_errs(ctx, ctx->m2l_err_flags);
  ctx->m2l_err_flags.clear();
  for (int i = 0; i < FMMA_NUM_STAGES; ++i) {
    if (!ctx->ev_used[i]) continue;
    float ms = 0.f;
    FMMA_CHECK_CUDA(cudaEventElapsedTime(&ms, ctx->ev[2 * i], ctx->ev[2 * i + 1]));
    ctx->stage_ms[i] = ms;
  }
}

// ---------------------------------------------------------------------------
// scan: 1024-element tiles, block sums scanned recursively
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanIpt = 4;
constexpr int kScanTile = kScanThreads * kScanIpt;

__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (int)(blockDim.x >> 5)) s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  int warp_off = warp > 0 ? s_warp[warp - 1] : 0;
  *total = s_warp[(blockDim.x >> 5) - 1];
  return warp_off + x - v;
}

__global__ void k_scan_tiles(const int* __restrict__ in, int* __restrict__ out, int64_t n,
                             int* __restrict__ block_sums) {
  __shared__ int s_warp[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanIpt;
  int v[kScanIpt];
  int tsum = 0;
#pragma unroll
  for (int i = 0; i < kScanIpt; ++i) {
    int64_t idx = base + i;
    v[i] = idx < n ? in[idx] : 0;
    tsum += v[i];
  }
  int total;
  int ex = block_exclusive_scan(tsum, s_warp, &total);
#pragma unroll
  for (int i = 0; i < kScanIpt; ++i) {
    int64_t idx = base + i;
    if (idx < n) out[idx] = ex;
    ex += v[i];
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int* __restrict__ out, int64_t n, const int* __restrict__ offs) {
  const int add = offs[blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
    int64_t idx = base + i;
    if (idx < n) out[idx] += add;
  }
}

// Short arrays (the coarse levels, the radix sort's digit offsets of small
// sorts) in one launch: one block walks the array in 4096-element tiles and
// carries the running total, and writes the total itself.
constexpr int kScanSmallThreads = 1024;
constexpr int64_t kScanSmallMax = 8192;

__global__ void __launch_bounds__(kScanSmallThreads) k_scan_small(const int* __restrict__ in, int* __restrict__ out,
                                                                  int64_t n, int* __restrict__ total_dev) {
  __shared__ int s_warp[32];
  int carry = 0;
  for (int64_t base = 0; base < n; base += (int64_t)kScanSmallThreads * kScanIpt) {
    const int64_t b = base + (int64_t)threadIdx.x * kScanIpt;
    int v[kScanIpt];
    int tsum = 0;
#pragma unroll
    for (int i = 0; i < kScanIpt; ++i) {
      v[i] = b + i < n ? in[b + i] : 0;
      tsum += v[i];
    }
    int total;
    int ex = carry + block_exclusive_scan(tsum, s_warp, &total);
#pragma unroll
    for (int i = 0; i < kScanIpt; ++i) {
      if (b + i < n) out[b + i] = ex;
      ex += v[i];
    }
    carry += total;
    __syncthreads();  // s_warp is rewritten by the next tile
  }
  if (threadIdx.x == 0) *total_dev = carry;
}

static void scan_rec(fmma_ctx* ctx, const int* in, int* out, int64_t n, int* total_dev, int depth) {
  if (n <= 0) {
    FMMA_CHECK_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(int), ctx->stream));
    return;
  }
  if (n <= kScanSmallMax) {
    FMMA_LAUNCH(ctx, k_scan_small, 1, kScanSmallThreads, 0, in, out, n, total_dev);
    return;
  }
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  int* bs = ctx_buf_t<int>(ctx, "scan_bs" + std::to_string(depth), (size_t)nb);
  FMMA_LAUNCH(ctx, k_scan_tiles, (unsigned)nb, kScanThreads, 0, in, out, n, bs);
  int* bo = ctx_buf_t<int>(ctx, "scan_bo" + std::to_string(depth), (size_t)nb);
  scan_rec(ctx, bs, bo, nb, total_dev, depth + 1);
  FMMA_LAUNCH(ctx, k_scan_add, (unsigned)nb, kScanThreads, 0, out, n, bo);
}

void scan_exclusive(fmma_ctx* ctx, const int* in, int* out, int64_t n, int* total_dev) {
  scan_rec(ctx, in, out, n, total_dev, 0);
}

// ---------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;
constexpr int kRsWarps = kRsThreads / 32;

__global__ void k_rs_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                          int* __restrict__ ghist, int nblocks) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int r = 0; r < kRsRounds; ++r) {
    int64_t e = base + (int64_t)r * kRsThreads + threadIdx.x;
    if (e < n) atomicAdd(&h[(int)((keys[e] >> shift) & 0xFF)], 1);
  }
  __syncthreads();
  ghist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Each round scatters 256 consecutive elements; ranks inside the round come
// from warp match masks and per-warp digit counts, so equal digits keep their
// input order (stability).
__global__ void k_rs_scatter(const uint64_t* __restrict__ kin, const int* __restrict__ vin,
                             uint64_t* __restrict__ kout, int* __restrict__ vout, int64_t n,
                             int shift, const int* __restrict__ goff, int nblocks) {
  __shared__ int running[256];
  __shared__ int wcnt[kRsWarps][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  running[tid] = goff[(int64_t)tid * nblocks + blockIdx.x];
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int r = 0; r < kRsRounds; ++r) {
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    int64_t e = base + (int64_t)r * kRsThreads + tid;
    bool valid = e < n;
    uint64_t k = valid ? kin[e] : 0ull;
    int v = valid ? vin[e] : 0;
    int dig = valid ? (int)((k >> shift) & 0xFF) : 256;
    unsigned m = __match_any_sync(0xffffffffu, dig);
    int rank = __popc(m & lt);
    if (valid && rank == 0) wcnt[warp][dig] = __popc(m);
    __syncthreads();
    {
      int acc = running[tid];
#pragma unroll
      for (int w = 0; w < kRsWarps; ++w) {
        int t = wcnt[w][tid];
        wcnt[w][tid] = acc;
        acc += t;
      }
      running[tid] = acc;
    }
    __syncthreads();
    if (valid) {
      int pos = wcnt[warp][dig] + rank;
      kout[pos] = k;
      vout[pos] = v;
    }
    __syncthreads();
  }
}

void radix_sort_pairs(fmma_ctx* ctx, uint64_t* keys, int* vals, int64_t n, int bit0, int bit1) {
  if (n <= 1 || bit1 <= bit0) return;
  int64_t nb64 = (n + kRsTile - 1) / kRsTile;
  int nb = (int)nb64;
  uint64_t* k2 = ctx_buf_t<uint64_t>(ctx, "rs_k2", (size_t)n);
  int* v2 = ctx_buf_t<int>(ctx, "rs_v2", (size_t)n);
  int* gh = ctx_buf_t<int>(ctx, "rs_hist", (size_t)256 * nb);
  int* go = ctx_buf_t<int>(ctx, "rs_off", (size_t)256 * nb);
  int* tot = ctx_buf_t<int>(ctx, "rs_tot", 1);
  uint64_t* ka = keys;
  int* va = vals;
  uint64_t* kb = k2;
  int* vb = v2;
  int passes = 0;
  for (int shift = bit0; shift < bit1; shift += 8) {
    FMMA_LAUNCH(ctx, k_rs_hist, nb, kRsThreads, 0, ka, n, shift, gh, nb);
    scan_exclusive(ctx, gh, go, (int64_t)256 * nb, tot);
    FMMA_LAUNCH(ctx, k_rs_scatter, nb, kRsThreads, 0, ka, va, kb, vb, n, shift, go, nb);
    std::swap(ka, kb);
    std::swap(va, vb);
    ++passes;
  }
  if (passes & 1) {
    FMMA_CHECK_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    FMMA_CHECK_CUDA(cudaMemcpyAsync(vals, va, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
  }
}

}  // namespace fmma_b200
