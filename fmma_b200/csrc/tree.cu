// tree.cu — integer tree build on the device: bounding cube, leaf binning
// (bit-exact with the reference), Morton keys, stable radix sort, leaf ranges,
// per-level box arrays, far (M2L) and near (P2P) interaction lists.
//
// Reference: binning src/fmm_core.cpp:255-267 and src/fmm.cpp:126-131, cube
// src/fmm_core.cpp:125-173, far list src/fmm_core.cpp:15-63, near list
// src/fmm_core.cpp:79-115.  The reference walks a dense 2^(d*l) grid; here
// only non-empty boxes exist (a box without sources contributes exact zeros
// to M2L/M2M/P2P, a box without targets receives nothing that is read).
#include <algorithm>
#include <cstring>

#include "fmm_stages.cuh"
#include "fmma_internal.cuh"

namespace fmma_b200 {

// ---------------------------------------------------------------------------
// far-slot tables
// ---------------------------------------------------------------------------
static FarTables g_far[kMaxDim + 1];
static bool g_far_init[kMaxDim + 1] = {false, false, false, false};

const FarTables& far_tables(int d) {
  FarTables& F = g_far[d];
  if (g_far_init[d]) return F;
  std::memset(&F, 0, sizeof(F));
  int p7 = 1, p6 = 1, p3 = 1;
  for (int q = 0; q < d; ++q) { p7 *= 7; p6 *= 6; p3 *= 3; }
  F.nfar = p6 - p3;
  F.noff = p7 - p3;
  F.nclass = 1 << d;
  // far offsets, row-major over (o + 3), last dimension fastest
  int offid[343];
  int cnt = 0;
  for (int s = 0; s < p7; ++s) {
    int o[3] = {0, 0, 0}, sc = s, dist = 0;
    for (int q = d - 1; q >= 0; --q) { o[q] = sc % 7 - 3; sc /= 7; dist = std::max(dist, std::abs(o[q])); }
    if (dist <= 1) { offid[s] = -1; continue; }
    offid[s] = cnt;
    for (int q = 0; q < d; ++q) F.off_vec[cnt][q] = o[q];
    ++cnt;
  }
  for (int c = 0; c < 8; ++c)
    for (int j = 0; j < 216; ++j) F.jslot[c][j] = -1;
  for (int c = 0; c < F.nclass; ++c) {
    int par[3] = {0, 0, 0};
    for (int q = 0; q < d; ++q) par[q] = (c >> (d - 1 - q)) & 1;
    int k = 0;
    for (int j = 0; j < p6; ++j) {
      int jd[3] = {0, 0, 0}, jc = j, dist = 0;
      for (int q = d - 1; q >= 0; --q) { jd[q] = jc % 6; jc /= 6; }
      int s7 = 0;
      for (int q = 0; q < d; ++q) {
        int o = jd[q] - 2 - par[q];
        dist = std::max(dist, std::abs(o));
        s7 = s7 * 7 + (o + 3);
      }
      if (dist <= 1) continue;
      F.slot_j[c][k] = j;
      F.slot_off[c][k] = offid[s7];
      F.jslot[c][j] = k;
      ++k;
    }
  }
  g_far_init[d] = true;
  return F;
}

// ---------------------------------------------------------------------------
// problem of each point, bounding cube per problem
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ord_enc(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_dec(unsigned long long u) {
  u = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double((long long)u);
}

__device__ __forceinline__ int find_seg(const int64_t* __restrict__ off, int np, int64_t i) {
  int lo = 0, hi = np;  // last p with off[p] <= i
  while (hi - lo > 1) {
    int m = (lo + hi) >> 1;
    if (off[m] <= i) lo = m; else hi = m;
  }
  return lo;
}

// problem id of each element of [targets | sources]
__global__ void k_point_pid(const int64_t* __restrict__ toff, const int64_t* __restrict__ soff, int np, int64_t nt,
                            int64_t ns, int* __restrict__ pid) {
  const int64_t n = nt + ns;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    pid[i] = np == 1 ? 0 : (i < nt ? find_seg(toff, np, i) : find_seg(soff, np, i - nt));
}

__global__ void k_bbox_init(unsigned long long* mm, int np, int* flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np * kMaxDim; i += gridDim.x * blockDim.x) {
    int p = i / kMaxDim, q = i % kMaxDim;
    mm[p * 2 * kMaxDim + q] = ~0ull;
    mm[p * 2 * kMaxDim + kMaxDim + q] = 0ull;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *flag = 0;
}

// Per-problem min/max of every coordinate over targets and sources: order
// free and exact (src/fmm_core.cpp:125-148).  Each warp scans one contiguous
// chunk (coalesced, 32 points per step) and each lane keeps running extrema
// for the problem it is in, flushing them with atomics only when the
// problem changes and once at the end (a warp reduction when the whole warp
// ends in one problem): a handful of atomics per warp instead of one per
// step.
__device__ __forceinline__ void bbox_flush(unsigned long long* mm, int p, int d, const unsigned long long* lo,
                                           const unsigned long long* hi) {
  for (int q = 0; q < d; ++q) {
    atomicMin(&mm[p * 2 * kMaxDim + q], lo[q]);
    atomicMax(&mm[p * 2 * kMaxDim + kMaxDim + q], hi[q]);
  }
}

template <typename T>
__global__ void k_bbox(const T* __restrict__ tgt, int64_t nt, const T* __restrict__ src, int64_t ns,
                       const int* __restrict__ pid, int d, unsigned long long* mm, int* flag) {
  const int64_t n = nt + ns;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t chunk = ((n + nw - 1) / nw + 31) / 32 * 32;
  const int64_t b0 = wid * chunk, b1 = min(n, b0 + chunk);
  int bad = 0, cur = -1;
  unsigned long long lo[kMaxDim], hi[kMaxDim];
  for (int q = 0; q < kMaxDim; ++q) { lo[q] = ~0ull; hi[q] = 0ull; }
  for (int64_t i = b0 + lane; i < b1; i += 32) {
    const int p = pid[i];
    if (p != cur) {
      if (cur >= 0) bbox_flush(mm, cur, d, lo, hi);
      for (int q = 0; q < kMaxDim; ++q) { lo[q] = ~0ull; hi[q] = 0ull; }
      cur = p;
    }
    const T* x = i < nt ? tgt + i * d : src + (i - nt) * d;
    for (int q = 0; q < d; ++q) {
      const double v = (double)x[q];
      if (!isfinite(v)) bad = 1;
      const unsigned long long e = ord_enc(v);
      lo[q] = e < lo[q] ? e : lo[q];
      hi[q] = e > hi[q] ? e : hi[q];
    }
  }
  const unsigned same = __match_any_sync(0xffffffffu, cur);
  if (same == 0xffffffffu) {
    for (int q = 0; q < d; ++q)
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[q], o);
        const unsigned long long bb = __shfl_xor_sync(0xffffffffu, hi[q], o);
        lo[q] = a < lo[q] ? a : lo[q];
        hi[q] = bb > hi[q] ? bb : hi[q];
      }
    if (lane == 0 && cur >= 0) bbox_flush(mm, cur, d, lo, hi);
  } else if (cur >= 0) {
    bbox_flush(mm, cur, d, lo, hi);
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0 && bad) atomicOr(flag, 1);
}

// src/fmm_core.cpp:160-173 in the caller's precision, one problem per thread.
// A degenerate cube (every coordinate equal: the reference divides by zero
// there) gets Len = 1.
__global__ void k_cube(const unsigned long long* mm, const int* flag, int np, int d, Cube* cubes) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const unsigned long long* m = mm + p * 2 * kMaxDim;
  double mn[kMaxDim], mx[kMaxDim];
  for (int q = 0; q < d; ++q) { mn[q] = ord_dec(m[q]); mx[q] = ord_dec(m[kMaxDim + q]); }
  Cube c;
  double L = 0.0;
  for (int q = 0; q < d; ++q) { double e = __dsub_rn(mx[q], mn[q]); L = L < e ? e : L; }
  if (!(L > 0.0)) L = 1.0;
  for (int q = 0; q < d; ++q) c.origin[q] = __dsub_rn(__dmul_rn(__dadd_rn(mx[q], mn[q]), 0.5), __dmul_rn(L, 0.5));
  c.Len = L;
  float Lf = 0.f;
  for (int q = 0; q < d; ++q) { float e = __fsub_rn((float)mx[q], (float)mn[q]); Lf = Lf < e ? e : Lf; }
  if (!(Lf > 0.f)) Lf = 1.f;
  for (int q = 0; q < d; ++q)
    c.originf[q] = __fsub_rn(__fmul_rn(__fadd_rn((float)mx[q], (float)mn[q]), 0.5f), __fmul_rn(Lf, 0.5f));
  c.Lenf = Lf;
  for (int q = d; q < kMaxDim; ++q) { c.origin[q] = 0.0; c.originf[q] = 0.f; }
  c.nonfinite = *flag;
  c.pad = 0;
  cubes[p] = c;
}

template <typename T>
__global__ void k_leaf_keys(const T* __restrict__ tgt, int64_t nt, const T* __restrict__ src, int64_t ns,
                            const int* __restrict__ pid, int d, const int* __restrict__ depth,
                            const Cube* __restrict__ cubes, uint64_t* __restrict__ keys, int* __restrict__ idx) {
  const int64_t n = nt + ns;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int p = pid[i];
    const Cube& c = cubes[p];
    const int bits = depth[p] - 1;
    const int N = 1 << bits;
    const T* x = i < nt ? tgt + i * d : src + (i - nt) * d;
    int cc[kMaxDim] = {0, 0, 0};
    for (int q = 0; q < d; ++q) cc[q] = bin_coord<T>(x[q], c, q, N);
    keys[i] = ((uint64_t)p << kPidShift) | morton_encode(cc, d, bits);
    if (idx) idx[i] = (int)i;
  }
}

// ---------------------------------------------------------------------------
// leaves and levels
// ---------------------------------------------------------------------------
__global__ void k_leaf_flags(const uint64_t* __restrict__ keys, const int* __restrict__ idx, int64_t n,
                             int64_t nt, int* __restrict__ fbox, int* __restrict__ ft) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    fbox[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
    ft[i] = idx[i] < nt ? 1 : 0;
  }
}

__global__ void k_leaf_emit(const uint64_t* __restrict__ keys, const int* __restrict__ idx, int64_t n,
                            int64_t nt, const int* __restrict__ fbox, const int* __restrict__ boxex,
                            const int* __restrict__ tex, int* __restrict__ perm_t,
                            int* __restrict__ perm_s, uint64_t* __restrict__ lkey,
                            int* __restrict__ ltb, int* __restrict__ lsb) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int id = idx[i];
    int tpos = tex[i];
    int spos = (int)i - tpos;
    if (id < nt) perm_t[tpos] = id;
    else perm_s[spos] = id - (int)nt;
    if (fbox[i]) {
      int b = boxex[i];
      lkey[b] = keys[i];
      ltb[b] = tpos;
      lsb[b] = spos;
    }
  }
}

__global__ void k_leaf_ends(int64_t nb, const int* __restrict__ tb, const int* __restrict__ sb,
                            int nt, int ns, int* __restrict__ te, int* __restrict__ se) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    te[b] = b + 1 < nb ? tb[b + 1] : nt;
    se[b] = b + 1 < nb ? sb[b + 1] : ns;
  }
}

__device__ __forceinline__ uint64_t parent_key(uint64_t k, int d) {
  return (k & ~kMortonMask) | ((k & kMortonMask) >> d);
}
__device__ __forceinline__ int real_level(uint64_t k, const int* depth, int v) {
  return depth[key_pid(k)] - 1 - v;
}

// A box of virtual level v has a parent when its real level is >= 1.
__global__ void k_parent_flags(const uint64_t* __restrict__ ckey, int64_t nc, int d, int v,
                               const int* __restrict__ depth, int* __restrict__ f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ckey[i];
    const bool valid = real_level(k, depth, v) >= 1;
    bool first = valid;
    if (valid && i > 0) {
      const uint64_t kp = ckey[i - 1];
      first = real_level(kp, depth, v) < 1 || parent_key(kp, d) != parent_key(k, d);
    }
    f[i] = first ? 1 : 0;
  }
}

// Box counts of every virtual level from key-sorted keys in one pass.  Key i
// opens a new box at virtual level v when its level-v ancestor differs from
// key i-1's: at every level v <= hb / d, hb the highest bit in which the two
// Morton codes differ, and at every level when the problem changes.  Levels
// stop at the problem's real level `cut` (virtual level depth - 1 - cut).
// hist[t] counts the keys whose highest new level is t, so level v holds
// sum_{t >= v} hist[t] boxes.  Two cuts at once: the points' keys give the
// boxes of every level (cut 0); the targets' keys give the boxes holding
// targets (cut 0: near-field rows) and those at real level >= 2 (cut 2: M2L
// rows).
__global__ void k_level_counts(const uint64_t* __restrict__ keys, int64_t n, int d,
                               const int* __restrict__ depth, int nlev, int cut_a, int* __restrict__ hist_a,
                               int cut_b, int* __restrict__ hist_b) {
  __shared__ int ha[32], hb[32];
  if (threadIdx.x < 32) {
    ha[threadIdx.x] = 0;
    hb[threadIdx.x] = 0;
  }
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const int p = key_pid(k);
    int diff = 63;  // highest level at which key i-1's ancestor differs
    if (i > 0) {
      const uint64_t kp = keys[i - 1];
      if (key_pid(kp) == p) {
        const uint64_t x = (k ^ kp) & kMortonMask;
        diff = x == 0 ? -1 : (63 - __clzll((long long)x)) / d;
      }
    }
    const int ta = min(diff, depth[p] - 1 - cut_a);
    if (ta >= 0) atomicAdd(&ha[ta], 1);
    if (hist_b) {
      const int tb = min(diff, depth[p] - 1 - cut_b);
      if (tb >= 0) atomicAdd(&hb[tb], 1);
    }
  }
  __syncthreads();
  if (threadIdx.x < nlev) {
    if (ha[threadIdx.x]) atomicAdd(&hist_a[threadIdx.x], ha[threadIdx.x]);
    if (hist_b && hb[threadIdx.x]) atomicAdd(&hist_b[threadIdx.x], hb[threadIdx.x]);
  }
}

// Keys of the targets in key order (position = exclusive target count).
__global__ void k_target_keys(const uint64_t* __restrict__ keys, const int* __restrict__ idx, int64_t n,
                              int64_t nt, const int* __restrict__ tex, uint64_t* __restrict__ tkey) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (idx[i] < nt) tkey[tex[i]] = keys[i];
}

// Parents of virtual level v.  pcap is the parent level's size, counted
// beforehand by k_level_counts; a parent index past it (which the counts rule
// out) raises *err instead of writing.
__global__ void k_parent_emit(const uint64_t* __restrict__ ckey, const int* __restrict__ ctb,
                              const int* __restrict__ cte, const int* __restrict__ csb,
                              const int* __restrict__ cse, int64_t nc, int d, int v,
                              const int* __restrict__ depth, const int* __restrict__ f,
                              const int* __restrict__ fex, int* __restrict__ cparent, uint64_t* __restrict__ pkey,
                              int* __restrict__ ptb, int* __restrict__ pte, int* __restrict__ psb,
                              int* __restrict__ pse, int* __restrict__ pcb, int* __restrict__ pce,
                              int64_t pcap, int* __restrict__ err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ckey[i];
    if (real_level(k, depth, v) < 1) {
      cparent[i] = -1;
      continue;
    }
    const int p = fex[i] + f[i] - 1;
    if (p < 0 || p >= pcap) {
      cparent[i] = -1;
      atomicExch(err, 1);
      continue;
    }
    cparent[i] = p;
    if (f[i]) {
      pkey[p] = parent_key(k, d);
      ptb[p] = ctb[i];
      psb[p] = csb[i];
      pcb[p] = (int)i;
    }
    const bool last = i == nc - 1 || f[i + 1] || real_level(ckey[i + 1], depth, v) < 1;
    if (last) {
      pte[p] = cte[i];
      pse[p] = cse[i];
      pce[p] = (int)i + 1;
    }
  }
}

// M2L rows: boxes with targets at real level >= 2, sort key (problem, class)
__global__ void k_row_flags(const uint64_t* __restrict__ key, const int* __restrict__ tb, const int* __restrict__ te,
                            int64_t nb, int v, int min_level, const int* __restrict__ depth, int* __restrict__ f) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x)
    f[b] = (te[b] > tb[b] && real_level(key[b], depth, v) >= min_level) ? 1 : 0;
}

__global__ void k_row_compact(const uint64_t* __restrict__ key, const int* __restrict__ f,
                              const int* __restrict__ fex, int64_t nb, int d,
                              uint64_t* __restrict__ ck, int* __restrict__ cv) {
  const uint64_t mask = (1ull << d) - 1ull;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (f[b]) {
      int r = fex[b];
      if (ck) ck[r] = ((uint64_t)key_pid(key[b]) << d) | (key[b] & mask);
      cv[r] = (int)b;
    }
  }
}

__global__ void k_seg_flags(const uint64_t* __restrict__ ck, int64_t n, int* __restrict__ f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    f[i] = (i == 0 || ck[i] != ck[i - 1]) ? 1 : 0;
}

// Segment table of one level at its slot of the table of all levels; cap is
// the slot's size (an upper bound of the level's segments; never exceeded).
__global__ void k_seg_emit(const uint64_t* __restrict__ ck, const int* __restrict__ f, const int* __restrict__ fex,
                           int64_t n, int cap, int* __restrict__ seg_key, int* __restrict__ seg_begin) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (f[i] && fex[i] < cap) {
      seg_key[fex[i]] = (int)ck[i];
      seg_begin[fex[i]] = (int)i;
    }
}

__global__ void k_pairs_p2p(const int* __restrict__ near, int64_t nrow, int nnear,
                            const int* __restrict__ row_box, const int* __restrict__ tb,
                            const int* __restrict__ te, const int* __restrict__ sb,
                            const int* __restrict__ se, unsigned long long* __restrict__ pairs) {
  unsigned long long mine = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrow;
       r += (int64_t)gridDim.x * blockDim.x) {
    int b = row_box[r];
    long long nsrc = 0;
    for (int q = 0; q < nnear; ++q) {
      int s = near[r * nnear + q];
      if (s >= 0) nsrc += se[s] - sb[s];
    }
    mine += (unsigned long long)nsrc * (unsigned long long)(te[b] - tb[b]);
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(pairs, mine);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
static int bits_for(int n) {
  int b = 0;
  while ((1 << b) < n) ++b;
  return b;
}

// Problem of every point and the cube of every problem (device and host).
template <typename T>
static void forest_cubes(fmma_ctx* ctx, int d, const std::vector<int64_t>& toff, const T* tgt,
                         const std::vector<int64_t>& soff, const T* src, Tree& tr, int* pid,
                         const char* cube_buf = "cube") {
  const int np = (int)toff.size() - 1;
  const int64_t nt = toff[(size_t)np], ns = soff[(size_t)np];
  int64_t* dto = ctx_buf_t<int64_t>(ctx, "forest_toff", (size_t)np + 1);
  int64_t* dso = ctx_buf_t<int64_t>(ctx, "forest_soff", (size_t)np + 1);
  upload(ctx, dto, toff.data(), sizeof(int64_t) * (size_t)(np + 1));
  upload(ctx, dso, soff.data(), sizeof(int64_t) * (size_t)(np + 1));
  FMMA_LAUNCH(ctx, k_point_pid, grid_for(nt + ns, 256, (int64_t)ctx->sm_count * 16), 256, 0, dto, dso, np, nt, ns, pid);
  unsigned long long* mm = ctx_buf_t<unsigned long long>(ctx, "bbox_mm", (size_t)np * 2 * kMaxDim);
  int* flag = ctx_buf_t<int>(ctx, "bbox_flag", 1);
  FMMA_LAUNCH(ctx, k_bbox_init, grid_for((int64_t)np * kMaxDim, 256), 256, 0, mm, np, flag);
  FMMA_LAUNCH(ctx, (k_bbox<T>), grid_for(nt + ns, 256, (int64_t)ctx->sm_count * 8), 256, 0, tgt, nt, src, ns, pid, d,
              mm, flag);
  tr.d_cube = static_cast<Cube*>(ctx_buf(ctx, cube_buf, sizeof(Cube) * (size_t)np));
  FMMA_LAUNCH(ctx, k_cube, grid_for(np, 128), 128, 0, mm, flag, np, d, tr.d_cube);
  tr.h_cube.resize((size_t)np);
  Cube* hp = static_cast<Cube*>(ctx_pinned(ctx, sizeof(Cube) * (size_t)np));
  FMMA_CHECK_CUDA(cudaMemcpyAsync(hp, tr.d_cube, sizeof(Cube) * (size_t)np, cudaMemcpyDeviceToHost, ctx->stream));
  FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(tr.h_cube.data(), hp, sizeof(Cube) * (size_t)np);
  if (tr.h_cube[0].nonfinite) throw Error(FMMA_ERR_INVALID_ARG, "a coordinate is NaN or Inf");
}

static void alloc_level(fmma_ctx* ctx, Level& L, int v, int64_t nb) {
  std::string s = "lev" + std::to_string(v) + "_";
  L.v = v;
  L.nbox = nb;
  const size_t n = (size_t)(nb > 0 ? nb : 1);
  L.key = ctx_buf_t<uint64_t>(ctx, s + "key", n);
  L.tb = ctx_buf_t<int>(ctx, s + "tb", n);
  L.te = ctx_buf_t<int>(ctx, s + "te", n);
  L.sb = ctx_buf_t<int>(ctx, s + "sb", n);
  L.se = ctx_buf_t<int>(ctx, s + "se", n);
  L.cb = ctx_buf_t<int>(ctx, s + "cb", n);
  L.ce = ctx_buf_t<int>(ctx, s + "ce", n);
  L.parent = ctx_buf_t<int>(ctx, s + "parent", n);
}

// Leaf keys, sorted; leaves; all virtual levels (no lists).
template <typename T>
static void forest_levels(fmma_ctx* ctx, int d, const std::vector<int64_t>& toff, const T* tgt,
                          const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth) {
  Tree& tr = ctx->tree;
  const int np = (int)depth.size();
  FMMA_REQUIRE(np >= 1 && np <= kMaxProblems, "between 1 and 4096 problems");
  FMMA_REQUIRE((int)toff.size() == np + 1 && (int)soff.size() == np + 1, "bad offsets");
  tr.valid = false;
  tr.d_pairs = nullptr;
  tr.pairs_read = true;
  tr.dim = d;
  tr.nprob = np;
  tr.depth = depth;
  tr.vmax = 0;
  for (int p = 0; p < np; ++p) {
    FMMA_REQUIRE(depth[(size_t)p] >= 1 && d * (depth[(size_t)p] - 1) <= kPidShift && depth[(size_t)p] - 1 <= 30,
                 "Depth out of range");
    tr.vmax = std::max(tr.vmax, depth[(size_t)p]);
  }
  tr.nt = toff[(size_t)np];
  tr.ns = soff[(size_t)np];
  const int64_t nt = tr.nt, ns = tr.ns, n = nt + ns;
  tr.lev.assign((size_t)tr.vmax, Level());
  tr.d_depth = ctx_buf_t<int>(ctx, "forest_depth", (size_t)np);
  upload(ctx, tr.d_depth, depth.data(), sizeof(int) * (size_t)np);
  const int blk = 256;
  const unsigned g = grid_for(n, blk, (int64_t)ctx->sm_count * 16);

  int* pid = ctx_buf_t<int>(ctx, "pt_pid", (size_t)(n > 0 ? n : 1));
  forest_cubes<T>(ctx, d, toff, tgt, soff, src, tr, pid);

  uint64_t* keys = ctx_buf_t<uint64_t>(ctx, "pt_keys", (size_t)n);
  int* idx = ctx_buf_t<int>(ctx, "pt_idx", (size_t)n);
  FMMA_LAUNCH(ctx, (k_leaf_keys<T>), g, blk, 0, tgt, nt, src, ns, pid, d, tr.d_depth, tr.d_cube, keys, idx);
  radix_sort_pairs(ctx, keys, idx, n, 0, d * (tr.vmax - 1));
  if (np > 1) radix_sort_pairs(ctx, keys, idx, n, kPidShift, kPidShift + bits_for(np));

  int* fbox = ctx_buf_t<int>(ctx, "pt_fbox", (size_t)n);
  int* ft = ctx_buf_t<int>(ctx, "pt_ft", (size_t)n);
  int* boxex = ctx_buf_t<int>(ctx, "pt_boxex", (size_t)n);
  int* tex = ctx_buf_t<int>(ctx, "pt_tex", (size_t)n);
  int* tot = ctx_buf_t<int>(ctx, "tree_tot", 4);
  FMMA_LAUNCH(ctx, k_leaf_flags, g, blk, 0, keys, idx, n, nt, fbox, ft);
  scan_exclusive(ctx, fbox, boxex, n, tot);
  scan_exclusive(ctx, ft, tex, n, tot + 1);
  // Sizes of every level and of the row sets of the lists, counted from the
  // sorted keys and read back in one wait: [0, V) boxes, [V, 2V) boxes with
  // targets, [2V, 3V) M2L rows (boxes with targets at real level >= 2), then
  // the leaf count of the scan as a check.
  const int V = tr.vmax;
  FMMA_REQUIRE(V <= 32, "Depth out of range");
  int* lvc = ctx_buf_t<int>(ctx, "tree_lvc", (size_t)3 * V + 1);
  FMMA_CHECK_CUDA(cudaMemsetAsync(lvc, 0, sizeof(int) * (size_t)3 * V, ctx->stream));
  FMMA_LAUNCH(ctx, k_level_counts, g, blk, 0, keys, n, d, tr.d_depth, V, 0, lvc, 0, (int*)nullptr);
  uint64_t* tkey = ctx_buf_t<uint64_t>(ctx, "pt_tkey", (size_t)(nt > 0 ? nt : 1));
  FMMA_LAUNCH(ctx, k_target_keys, g, blk, 0, keys, idx, n, nt, tex, tkey);
  FMMA_LAUNCH(ctx, k_level_counts, grid_for(nt, blk, (int64_t)ctx->sm_count * 16), blk, 0, tkey, nt, d, tr.d_depth,
              V, 0, lvc + V, 2, lvc + 2 * V);
  FMMA_CHECK_CUDA(cudaMemcpyAsync(lvc + 3 * V, tot, sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
  std::vector<int> hl((size_t)3 * V + 1, 0);
  read_ints(ctx, lvc, hl.data(), 3 * V + 1);
  for (int c = 0; c < 3; ++c)  // histogram of highest new level -> boxes per level
    for (int v = V - 2; v >= 0; --v) hl[(size_t)(c * V + v)] += hl[(size_t)(c * V + v + 1)];
  const int64_t nleaf = hl[(size_t)3 * V];
  if (hl[0] != nleaf) throw Error(FMMA_ERR_CUDA, "tree build: level counts disagree with the leaf scan");
  tr.near_count = hl[(size_t)V];
  tr.row_count.assign(hl.begin() + 2 * V, hl.begin() + 3 * V);
  tr.d_err = ctx_buf_t<int>(ctx, "tree_err", 1);
  FMMA_CHECK_CUDA(cudaMemsetAsync(tr.d_err, 0, sizeof(int), ctx->stream));

  tr.perm_t = ctx_buf_t<int>(ctx, "perm_t", (size_t)(nt > 0 ? nt : 1));
  tr.perm_s = ctx_buf_t<int>(ctx, "perm_s", (size_t)(ns > 0 ? ns : 1));
  Level& leaf = tr.lev[0];
  alloc_level(ctx, leaf, 0, nleaf);
  FMMA_LAUNCH(ctx, k_leaf_emit, g, blk, 0, keys, idx, n, nt, fbox, boxex, tex, tr.perm_t, tr.perm_s, leaf.key,
              leaf.tb, leaf.sb);
  FMMA_LAUNCH(ctx, k_leaf_ends, grid_for(nleaf, blk), blk, 0, nleaf, leaf.tb, leaf.sb, (int)nt, (int)ns, leaf.te,
              leaf.se);
  FMMA_CHECK_CUDA(cudaMemsetAsync(leaf.cb, 0, sizeof(int) * (size_t)nleaf, ctx->stream));
  FMMA_CHECK_CUDA(cudaMemsetAsync(leaf.ce, 0, sizeof(int) * (size_t)nleaf, ctx->stream));

  for (int v = 0; v + 1 < tr.vmax; ++v) {
    Level& C = tr.lev[(size_t)v];
    int* f = ctx_buf_t<int>(ctx, "lv_f", (size_t)C.nbox + 1);
    int* fex = ctx_buf_t<int>(ctx, "lv_fex", (size_t)C.nbox + 1);
    FMMA_LAUNCH(ctx, k_parent_flags, grid_for(C.nbox, blk), blk, 0, C.key, C.nbox, d, v, tr.d_depth, f);
    scan_exclusive(ctx, f, fex, C.nbox, tot);
    Level& Pl = tr.lev[(size_t)(v + 1)];
    alloc_level(ctx, Pl, v + 1, hl[(size_t)(v + 1)]);
    FMMA_LAUNCH(ctx, k_parent_emit, grid_for(C.nbox, blk), blk, 0, C.key, C.tb, C.te, C.sb, C.se, C.nbox, d, v,
                tr.d_depth, f, fex, C.parent, Pl.key, Pl.tb, Pl.te, Pl.sb, Pl.se, Pl.cb, Pl.ce, Pl.nbox, tr.d_err);
  }
  Level& top = tr.lev[(size_t)(tr.vmax - 1)];
  FMMA_CHECK_CUDA(cudaMemsetAsync(top.parent, 0xff, sizeof(int) * (size_t)(top.nbox > 0 ? top.nbox : 1), ctx->stream));
}

template <typename T>
void build_forest(fmma_ctx* ctx, int d, const std::vector<int64_t>& toff, const T* tgt,
                  const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth, bool lists) {
  forest_levels<T>(ctx, d, toff, tgt, soff, src, depth);
  Tree& tr = ctx->tree;
  const int np = tr.nprob;
  const int blk = 256;
  if (lists) {
    const FarTables& F = far_tables(d);
    int* jslot = ctx_buf_t<int>(ctx, "jslot", 8 * 216);
    upload(ctx, jslot, F.jslot, sizeof(int) * 8 * 216);
    unsigned long long* pairs = ctx_buf_t<unsigned long long>(ctx, "il_pairs", (size_t)tr.vmax + 2);
    FMMA_CHECK_CUDA(cudaMemsetAsync(pairs, 0, sizeof(unsigned long long) * (size_t)(tr.vmax + 2), ctx->stream));
    const int pbits = bits_for(np);
    const int V = tr.vmax;
    // The row counts come from the level counts; the host waits on the device
    // once for the segment tables of all levels and once for the pair counts.
    // cnt receives the row scans' totals (unused: the counts are known).
    int* cnt = ctx_buf_t<int>(ctx, "tree_cnt", (size_t)V + 1);
    std::vector<int*> fv((size_t)V, nullptr), fexv((size_t)V, nullptr);
    for (int v = 0; v < V; ++v) {
      Level& Lv = tr.lev[(size_t)v];
      // operator tables: problems with a real level >= 2 at this virtual level
      Lv.pid_table.assign((size_t)np, -1);
      Lv.table_pid.clear();
      for (int p = 0; p < np; ++p)
        if (tr.depth[(size_t)p] - 1 - v >= 2) {
          Lv.pid_table[(size_t)p] = (int)Lv.table_pid.size();
          Lv.table_pid.push_back(p);
        }
      Lv.nrow = 0;
      Lv.segs.clear();
      if (Lv.table_pid.empty()) continue;
      fv[(size_t)v] = ctx_buf_t<int>(ctx, "lv_f" + std::to_string(v), (size_t)Lv.nbox + 1);
      fexv[(size_t)v] = ctx_buf_t<int>(ctx, "lv_fex" + std::to_string(v), (size_t)Lv.nbox + 1);
      FMMA_LAUNCH(ctx, k_row_flags, grid_for(Lv.nbox, blk), blk, 0, Lv.key, Lv.tb, Lv.te, Lv.nbox, v, 2, tr.d_depth,
                  fv[(size_t)v]);
      scan_exclusive(ctx, fv[(size_t)v], fexv[(size_t)v], Lv.nbox, cnt + v);
    }
    int* fnear = ctx_buf_t<int>(ctx, "near_f", (size_t)tr.lev[0].nbox + 1);
    int* fexnear = ctx_buf_t<int>(ctx, "near_fex", (size_t)tr.lev[0].nbox + 1);
    FMMA_LAUNCH(ctx, k_row_flags, grid_for(tr.lev[0].nbox, blk), blk, 0, tr.lev[0].key, tr.lev[0].tb, tr.lev[0].te,
                tr.lev[0].nbox, 0, 0, tr.d_depth, fnear);
    scan_exclusive(ctx, fnear, fexnear, tr.lev[0].nbox, cnt + V);
    // rows per level and near rows were counted with the levels
    std::vector<int> hc((size_t)2 * V + 2, 0);
    for (int v = 0; v < V; ++v) hc[(size_t)v] = tr.lev[(size_t)v].table_pid.empty() ? 0 : tr.row_count[(size_t)v];
    hc[(size_t)V] = (int)tr.near_count;
    // Rows sorted by (problem, class) and each level's segment table, all read
    // back in one wait: seg_all = [segments per level (V) | keys | begins],
    // level v's table at sbo[v] with room for min(rows, problems x classes).
    std::vector<int> sbo((size_t)V + 1, 0);
    for (int v = 0; v < V; ++v)
      sbo[(size_t)v + 1] = sbo[(size_t)v] + (int)std::min<int64_t>(hc[(size_t)v], (int64_t)np << d);
    const int TB = sbo[(size_t)V];
    int* seg_all = ctx_buf_t<int>(ctx, "seg_all", (size_t)V + 2 * (size_t)TB);
    FMMA_CHECK_CUDA(cudaMemsetAsync(seg_all, 0, sizeof(int) * (size_t)V, ctx->stream));
    std::vector<uint64_t*> ckv((size_t)V, nullptr);
    std::vector<int*> sfv((size_t)V, nullptr), sfxv((size_t)V, nullptr);
    for (int v = 0; v < V; ++v) {
      Level& Lv = tr.lev[(size_t)v];
      if (Lv.table_pid.empty()) continue;
      const int nr = hc[(size_t)v];
      Lv.nrow = nr;
      std::string s = "lev" + std::to_string(v) + "_";
      ckv[(size_t)v] = ctx_buf_t<uint64_t>(ctx, s + "row_ck", (size_t)(nr > 0 ? nr : 1));
      Lv.row_box = ctx_buf_t<int>(ctx, s + "row_box", (size_t)(nr > 0 ? nr : 1));
      Lv.il = ctx_buf_t<int>(ctx, s + "il", (size_t)nr * F.nfar + 1);
      Lv.slot_mask = ctx_buf_t<unsigned>(ctx, s + "smask", (size_t)nr * kSlotWords + 1);
      if (nr == 0) continue;
      uint64_t* ck = ckv[(size_t)v];
      FMMA_LAUNCH(ctx, k_row_compact, grid_for(Lv.nbox, blk), blk, 0, Lv.key, fv[(size_t)v], fexv[(size_t)v], Lv.nbox,
                  d, ck, Lv.row_box);
      radix_sort_pairs(ctx, ck, Lv.row_box, nr, 0, d + pbits);
      sfv[(size_t)v] = ctx_buf_t<int>(ctx, s + "seg_f", (size_t)nr);
      sfxv[(size_t)v] = ctx_buf_t<int>(ctx, s + "seg_fex", (size_t)nr);
      FMMA_LAUNCH(ctx, k_seg_flags, grid_for(nr, blk), blk, 0, ck, (int64_t)nr, sfv[(size_t)v]);
      scan_exclusive(ctx, sfv[(size_t)v], sfxv[(size_t)v], nr, seg_all + v);
      const int cap = sbo[(size_t)v + 1] - sbo[(size_t)v];
      FMMA_LAUNCH(ctx, k_seg_emit, grid_for(nr, blk), blk, 0, ck, sfv[(size_t)v], sfxv[(size_t)v], (int64_t)nr, cap,
                  seg_all + V + sbo[(size_t)v], seg_all + V + TB + sbo[(size_t)v]);
    }
    std::vector<int> hseg((size_t)V + 2 * (size_t)TB);
    read_ints(ctx, seg_all, hseg.data(), V + 2 * TB);
    for (int v = 0; v < V; ++v) {
      Level& Lv = tr.lev[(size_t)v];
      const int nseg = hseg[(size_t)v];
      if (nseg > sbo[(size_t)v + 1] - sbo[(size_t)v])
        throw Error(FMMA_ERR_CUDA, "tree build: more row segments than (problem, class) pairs");
      const int* sk = hseg.data() + V + sbo[(size_t)v];
      const int* sb = hseg.data() + V + TB + sbo[(size_t)v];
      for (int i = 0; i < nseg; ++i)
        Lv.segs.push_back(make_int4(sk[i] >> d, sk[i] & ((1 << d) - 1), sb[i], i + 1 < nseg ? sb[i + 1] : (int)Lv.nrow));
    }
    // neighbour lists of every level top-down, far lists of the rows on the way
    const int nnb = d == 1 ? 3 : (d == 2 ? 9 : 27);
    int64_t maxbox = 1;
    for (const Level& L : tr.lev) maxbox = std::max<int64_t>(maxbox, L.nbox);
    int* nbr[2] = {ctx_buf_t<int>(ctx, "nbr_even", (size_t)maxbox * nnb),
                   ctx_buf_t<int>(ctx, "nbr_odd", (size_t)maxbox * nnb)};
    int* row_of = ctx_buf_t<int>(ctx, "row_of_box", (size_t)maxbox);
    for (int v = tr.vmax - 1; v >= 0; --v) {
      const bool top = v + 1 >= tr.vmax;
      launch_lists_topdown(ctx, tr.lev[(size_t)v], top ? nullptr : &tr.lev[(size_t)(v + 1)],
                           top ? nullptr : nbr[(v + 1) & 1], d, F.nfar, jslot, nbr[v & 1], row_of, pairs + v);
    }
    // near lists at the leaves (rows = leaves with targets, key order)
    {
      Level& Lv = tr.lev[0];
      const int nr = hc[(size_t)V];
      tr.nnear_rows = nr;
      const int nnear = d == 1 ? 3 : (d == 2 ? 9 : 27);
      tr.near_row_box = ctx_buf_t<int>(ctx, "near_row_box", (size_t)(nr > 0 ? nr : 1));
      tr.near = ctx_buf_t<int>(ctx, "near", (size_t)nr * nnear + 1);
      if (nr > 0) {
        FMMA_LAUNCH(ctx, k_row_compact, grid_for(Lv.nbox, blk), blk, 0, Lv.key, fnear, fexnear, Lv.nbox, d,
                    (uint64_t*)nullptr, tr.near_row_box);
        launch_near_rows(ctx, nbr[0], tr.near_row_box, (int64_t)nr, d, Lv.sb, Lv.se, tr.near);
        FMMA_LAUNCH(ctx, k_pairs_p2p, grid_for(nr, blk), blk, 0, tr.near, (int64_t)nr, nnear, tr.near_row_box, Lv.tb,
                    Lv.te, Lv.sb, Lv.se, pairs + tr.vmax);
      }
    }
    tr.d_pairs = pairs;  // read when needed (tree_read_pairs)
    tr.pairs_read = false;
  }
  tr.valid = true;
}

void tree_read_pairs(fmma_ctx* ctx) {
  Tree& tr = ctx->tree;
  if (tr.pairs_read || !tr.d_pairs) return;
  std::vector<unsigned long long> hp((size_t)tr.vmax + 1);
  unsigned long long* pp =
      static_cast<unsigned long long*>(ctx_pinned(ctx, sizeof(unsigned long long) * (hp.size() + 1)));
  FMMA_CHECK_CUDA(cudaMemcpyAsync(pp, tr.d_pairs, sizeof(unsigned long long) * hp.size(), cudaMemcpyDeviceToHost,
                                  ctx->stream));
  FMMA_CHECK_CUDA(cudaMemcpyAsync(pp + hp.size(), tr.d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(hp.data(), pp, sizeof(unsigned long long) * hp.size());
  int herr = 0;
  std::memcpy(&herr, pp + hp.size(), sizeof(int));
  tr.pairs_read = true;
  if (herr) throw Error(FMMA_ERR_CUDA, "tree build: a level holds more boxes than counted");
  for (int v = 0; v < tr.vmax; ++v) tr.lev[(size_t)v].il_pairs = (int64_t)hp[(size_t)v];
  tr.p2p_pairs = (int64_t)hp[(size_t)tr.vmax];
}

template void build_forest<double>(fmma_ctx*, int, const std::vector<int64_t>&, const double*,
                                   const std::vector<int64_t>&, const double*, const std::vector<int>&, bool);
template void build_forest<float>(fmma_ctx*, int, const std::vector<int64_t>&, const float*,
                                  const std::vector<int64_t>&, const float*, const std::vector<int>&, bool);

template <typename T>
void build_tree(fmma_ctx* ctx, int d, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src, bool lists) {
  build_forest<T>(ctx, d, {0, nt}, tgt, {0, ns}, src, {depth}, lists);
}

template void build_tree<double>(fmma_ctx*, int, int, int64_t, const double*, int64_t, const double*, bool);
template void build_tree<float>(fmma_ctx*, int, int, int64_t, const float*, int64_t, const float*, bool);

// ---------------------------------------------------------------------------
// occupancy and export
// ---------------------------------------------------------------------------
__global__ void k_max_run(const uint64_t* __restrict__ key, const int* __restrict__ tb, const int* __restrict__ te,
                          const int* __restrict__ sb, const int* __restrict__ se, int64_t nb, int* __restrict__ out) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int p = key_pid(key[b]);
    atomicMax(&out[2 * p], te[b] - tb[b]);
    atomicMax(&out[2 * p + 1], se[b] - sb[b]);
  }
}

template <typename T>
void leaf_occupancy(fmma_ctx* ctx, int d, const std::vector<int64_t>& toff, const T* tgt,
                    const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth,
                    std::vector<int>* max_t, std::vector<int>* max_s) {
  forest_levels<T>(ctx, d, toff, tgt, soff, src, depth);
  const int np = (int)depth.size();
  Level& leaf = ctx->tree.lev[0];
  int* out = ctx_buf_t<int>(ctx, "occ", (size_t)2 * np);
  FMMA_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(int) * 2 * (size_t)np, ctx->stream));
  FMMA_LAUNCH(ctx, k_max_run, grid_for(leaf.nbox, 256), 256, 0, leaf.key, leaf.tb, leaf.te, leaf.sb, leaf.se, leaf.nbox,
              out);
  std::vector<int> h((size_t)2 * np);
  read_ints(ctx, out, h.data(), 2 * np);
  max_t->resize((size_t)np);
  max_s->resize((size_t)np);
  for (int p = 0; p < np; ++p) {
    (*max_t)[(size_t)p] = h[(size_t)(2 * p)];
    (*max_s)[(size_t)p] = h[(size_t)(2 * p + 1)];
  }
  ctx->tree.valid = false;
}

template void leaf_occupancy<double>(fmma_ctx*, int, const std::vector<int64_t>&, const double*,
                                     const std::vector<int64_t>&, const double*, const std::vector<int>&,
                                     std::vector<int>*, std::vector<int>*);
template void leaf_occupancy<float>(fmma_ctx*, int, const std::vector<int64_t>&, const float*,
                                    const std::vector<int64_t>&, const float*, const std::vector<int>&,
                                    std::vector<int>*, std::vector<int>*);

__global__ void k_key_to_rowmajor(const uint64_t* __restrict__ keys, int64_t n, int d, int bits,
                                  int64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c[kMaxDim] = {0, 0, 0};
    morton_decode(keys[i] & kMortonMask, d, bits, c);
    int64_t r = 0;
    for (int q = 0; q < d; ++q) r = (r << bits) | (int64_t)c[q];
    out[i] = r;
  }
}

template <typename T>
void export_bins(fmma_ctx* ctx, int d, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src,
                 int64_t* tbox, int64_t* sbox, Cube* cube_out) {
  Tree tmp;
  const int64_t n = nt + ns;
  int* pid = ctx_buf_t<int>(ctx, "pt_pid", (size_t)(n > 0 ? n : 1));
  forest_cubes<T>(ctx, d, {0, nt}, tgt, {0, ns}, src, tmp, pid);
  *cube_out = tmp.h_cube[0];
  int* dd = ctx_buf_t<int>(ctx, "export_depth", 1);
  upload(ctx, dd, &depth, sizeof(int));
  uint64_t* keys = ctx_buf_t<uint64_t>(ctx, "pt_keys", (size_t)(n > 0 ? n : 1));
  const int bits = depth - 1;
  FMMA_LAUNCH(ctx, (k_leaf_keys<T>), grid_for(n, 256), 256, 0, tgt, nt, src, ns, pid, d, dd, tmp.d_cube, keys,
              (int*)nullptr);
  if (nt > 0) FMMA_LAUNCH(ctx, k_key_to_rowmajor, grid_for(nt, 256), 256, 0, keys, nt, d, bits, tbox);
  if (ns > 0) FMMA_LAUNCH(ctx, k_key_to_rowmajor, grid_for(ns, 256), 256, 0, keys + nt, ns, d, bits, sbox);
}

template <typename T>
const Cube* problem_cube(fmma_ctx* ctx, int d, int64_t nt, const T* tgt, int64_t ns, const T* src,
                         const char* cube_buf, Cube* host) {
  Tree tmp;
  const int64_t n = nt + ns;
  int* pid = ctx_buf_t<int>(ctx, "pt_pid", (size_t)(n > 0 ? n : 1));
  forest_cubes<T>(ctx, d, {0, nt}, tgt, {0, ns}, src, tmp, pid, cube_buf);
  *host = tmp.h_cube[0];
  return tmp.d_cube;
}

template const Cube* problem_cube<double>(fmma_ctx*, int, int64_t, const double*, int64_t, const double*, const char*,
                                          Cube*);
template const Cube* problem_cube<float>(fmma_ctx*, int, int64_t, const float*, int64_t, const float*, const char*,
                                         Cube*);

template void export_bins<double>(fmma_ctx*, int, int, int64_t, const double*, int64_t, const double*, int64_t*, int64_t*, Cube*);
template void export_bins<float>(fmma_ctx*, int, int, int64_t, const float*, int64_t, const float*, int64_t*, int64_t*, Cube*);

}  // namespace fmma_b200
