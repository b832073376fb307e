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
      ++k;
    }
  }
  g_far_init[d] = true;
  return F;
}

// ---------------------------------------------------------------------------
// bounding cube
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ord_enc(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_dec(unsigned long long u) {
  u = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double((long long)u);
}

__global__ void k_bbox_init(unsigned long long* mm, int* flag) {
  int t = threadIdx.x;
  if (t < kMaxDim) { mm[t] = ~0ull; mm[kMaxDim + t] = 0ull; }
  if (t == 0) *flag = 0;
}

template <typename T>
__global__ void k_bbox(const T* __restrict__ tgt, int64_t nt, const T* __restrict__ src, int64_t ns,
                       int d, unsigned long long* mm, int* flag) {
  unsigned long long lo[kMaxDim], hi[kMaxDim];
  for (int q = 0; q < kMaxDim; ++q) { lo[q] = ~0ull; hi[q] = 0ull; }
  int bad = 0;
  const int64_t n = nt + ns;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T* p = i < nt ? tgt + i * d : src + (i - nt) * d;
    for (int q = 0; q < d; ++q) {
      double v = (double)p[q];
      if (!isfinite(v)) bad = 1;
      unsigned long long e = ord_enc(v);
      lo[q] = e < lo[q] ? e : lo[q];
      hi[q] = e > hi[q] ? e : hi[q];
    }
  }
  for (int q = 0; q < d; ++q) {
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[q], o);
      unsigned long long b = __shfl_xor_sync(0xffffffffu, hi[q], o);
      lo[q] = a < lo[q] ? a : lo[q];
      hi[q] = b > hi[q] ? b : hi[q];
    }
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    for (int q = 0; q < d; ++q) {
      atomicMin(&mm[q], lo[q]);
      atomicMax(&mm[kMaxDim + q], hi[q]);
    }
    if (bad) atomicOr(flag, 1);
  }
}

// src/fmm_core.cpp:160-173 in the caller's precision.  A degenerate cube
// (every coordinate equal: the reference divides by zero there) gets Len=1.
__global__ void k_cube(const unsigned long long* mm, const int* flag, int d, Cube* cube) {
  double mn[kMaxDim], mx[kMaxDim];
  for (int q = 0; q < d; ++q) { mn[q] = ord_dec(mm[q]); mx[q] = ord_dec(mm[kMaxDim + q]); }
  double L = 0.0;
  for (int q = 0; q < d; ++q) { double e = __dsub_rn(mx[q], mn[q]); L = L < e ? e : L; }
  if (!(L > 0.0)) L = 1.0;
  for (int q = 0; q < d; ++q)
    cube->origin[q] = __dsub_rn(__dmul_rn(__dadd_rn(mx[q], mn[q]), 0.5), __dmul_rn(L, 0.5));
  cube->Len = L;
  float Lf = 0.f;
  for (int q = 0; q < d; ++q) {
    float e = __fsub_rn((float)mx[q], (float)mn[q]);
    Lf = Lf < e ? e : Lf;
  }
  if (!(Lf > 0.f)) Lf = 1.f;
  for (int q = 0; q < d; ++q)
    cube->originf[q] = __fsub_rn(__fmul_rn(__fadd_rn((float)mx[q], (float)mn[q]), 0.5f), __fmul_rn(Lf, 0.5f));
  cube->Lenf = Lf;
  for (int q = d; q < kMaxDim; ++q) { cube->origin[q] = 0.0; cube->originf[q] = 0.f; }
  cube->nonfinite = *flag;
}

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

template <typename T>
__global__ void k_leaf_keys(const T* __restrict__ tgt, int64_t nt, const T* __restrict__ src,
                            int64_t ns, int d, int bits, const Cube* __restrict__ cube,
                            uint64_t* __restrict__ keys, int* __restrict__ idx) {
  const Cube c = *cube;
  const int N = 1 << bits;
  const int64_t n = nt + ns;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T* p = i < nt ? tgt + i * d : src + (i - nt) * d;
    int cc[kMaxDim] = {0, 0, 0};
    for (int q = 0; q < d; ++q) cc[q] = bin_coord<T>(p[q], c, q, N);
    keys[i] = morton_encode(cc, d, bits);
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

__global__ void k_parent_flags(const uint64_t* __restrict__ ckey, int64_t nc, int d, int* __restrict__ f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x)
    f[i] = (i == 0 || (ckey[i] >> d) != (ckey[i - 1] >> d)) ? 1 : 0;
}

__global__ void k_parent_emit(const uint64_t* __restrict__ ckey, const int* __restrict__ ctb,
                              const int* __restrict__ cte, const int* __restrict__ csb,
                              const int* __restrict__ cse, int64_t nc, int d,
                              const int* __restrict__ f, const int* __restrict__ fex,
                              int* __restrict__ cparent, uint64_t* __restrict__ pkey,
                              int* __restrict__ ptb, int* __restrict__ pte, int* __restrict__ psb,
                              int* __restrict__ pse, int* __restrict__ pcb, int* __restrict__ pce) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    int p = fex[i] + f[i] - 1;
    cparent[i] = p;
    if (f[i]) {
      pkey[p] = ckey[i] >> d;
      ptb[p] = ctb[i];
      psb[p] = csb[i];
      pcb[p] = (int)i;
    }
    if (i == nc - 1 || f[i + 1]) {
      pte[p] = cte[i];
      pse[p] = cse[i];
      pce[p] = (int)i + 1;
    }
  }
}

__global__ void k_row_flags(const int* __restrict__ tb, const int* __restrict__ te, int64_t nb,
                            int* __restrict__ f) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x)
    f[b] = te[b] > tb[b] ? 1 : 0;
}

__global__ void k_row_compact(const uint64_t* __restrict__ key, const int* __restrict__ f,
                              const int* __restrict__ fex, int64_t nb, int d,
                              uint64_t* __restrict__ ck, int* __restrict__ cv) {
  const uint64_t mask = (1ull << d) - 1ull;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (f[b]) {
      int r = fex[b];
      if (ck) ck[r] = key[b] & mask;
      cv[r] = (int)b;
    }
  }
}

__global__ void k_class_bounds(const uint64_t* __restrict__ ck, int64_t n, int ncls, int* __restrict__ out) {
  int c = threadIdx.x;
  if (c > ncls) return;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if ((int)ck[m] < c) lo = m + 1; else hi = m;
  }
  out[c] = (int)lo;
}

__device__ __forceinline__ int find_box(const uint64_t* __restrict__ keys, int64_t nb, uint64_t k) {
  int64_t lo = 0, hi = nb;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (keys[m] < k) lo = m + 1; else hi = m;
  }
  return (lo < nb && keys[lo] == k) ? (int)lo : -1;
}

struct SlotTab {
  int slot_j[8][189];
};

__global__ void k_build_il(const uint64_t* __restrict__ key, const int* __restrict__ sb,
                           const int* __restrict__ se, int64_t nb, const int* __restrict__ row_box,
                           int64_t nrow, int d, int l, int nfar, const int* __restrict__ slot_j,
                           int* __restrict__ il, unsigned long long* __restrict__ pairs) {
  const int64_t total = nrow * nfar;
  const int N = 1 << l;
  const uint64_t cmask = (1ull << d) - 1ull;
  unsigned long long mine = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row = e / nfar;
    int q = (int)(e - row * nfar);
    int b = row_box[row];
    uint64_t k = key[b];
    int cls = (int)(k & cmask);
    int c[kMaxDim] = {0, 0, 0};
    morton_decode(k, d, l, c);
    int j = slot_j[cls * 189 + q];
    int pos[kMaxDim] = {0, 0, 0};
    bool in = true;
    for (int qq = d - 1; qq >= 0; --qq) {
      int jd = j % 6;
      j /= 6;
      pos[qq] = 2 * (c[qq] >> 1) - 2 + jd;
      in = in && pos[qq] >= 0 && pos[qq] < N;
    }
    int res = -1;
    if (in) {
      int bb = find_box(key, nb, morton_encode(pos, d, l));
      if (bb >= 0 && se[bb] > sb[bb]) res = bb;
    }
    il[e] = res;
    mine += res >= 0 ? 1ull : 0ull;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(pairs, mine);
}

// near list of each leaf row: clamped 3^d block, last dimension fastest
__global__ void k_build_near(const uint64_t* __restrict__ key, const int* __restrict__ sb,
                             const int* __restrict__ se, int64_t nb, const int* __restrict__ row_box,
                             int64_t nrow, int d, int l, int nnear, int* __restrict__ near) {
  const int64_t total = nrow * nnear;
  const int N = 1 << l;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row = e / nnear;
    int q = (int)(e - row * nnear);
    int b = row_box[row];
    int c[kMaxDim] = {0, 0, 0};
    morton_decode(key[b], d, l, c);
    int pos[kMaxDim] = {0, 0, 0};
    bool in = true;
    int qc = q;
    for (int qq = d - 1; qq >= 0; --qq) {
      pos[qq] = c[qq] + qc % 3 - 1;
      qc /= 3;
      in = in && pos[qq] >= 0 && pos[qq] < N;
    }
    int res = -1;
    if (in) {
      int bb = find_box(key, nb, morton_encode(pos, d, l));
      if (bb >= 0 && se[bb] > sb[bb]) res = bb;
    }
    near[e] = res;
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
template <typename T>
static Cube* compute_cube(fmma_ctx* ctx, int d, int64_t nt, const T* tgt, int64_t ns, const T* src) {
  unsigned long long* mm = ctx_buf_t<unsigned long long>(ctx, "bbox_mm", 2 * kMaxDim);
  int* flag = ctx_buf_t<int>(ctx, "bbox_flag", 1);
  Cube* cube = static_cast<Cube*>(ctx_buf(ctx, "cube", sizeof(Cube)));
  FMMA_LAUNCH(ctx, k_bbox_init, 1, 32, 0, mm, flag);
  FMMA_LAUNCH(ctx, (k_bbox<T>), grid_for(nt + ns, 256, (int64_t)ctx->sm_count * 8), 256, 0,
              tgt, nt, src, ns, d, mm, flag);
  FMMA_LAUNCH(ctx, k_cube, 1, 1, 0, mm, flag, d, cube);
  return cube;
}

static void check_cube(fmma_ctx* ctx, Cube* cube_dev, Cube* host) {
  Cube* p = static_cast<Cube*>(ctx_pinned(ctx, sizeof(Cube)));
  FMMA_CHECK_CUDA(cudaMemcpyAsync(p, cube_dev, sizeof(Cube), cudaMemcpyDeviceToHost, ctx->stream));
  FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  *host = *p;
  if (host->nonfinite) throw Error(FMMA_ERR_INVALID_ARG, "a coordinate is NaN or Inf");
}

static void alloc_level(fmma_ctx* ctx, Level& L, int l, int64_t nb) {
  std::string s = "lev" + std::to_string(l) + "_";
  L.nbox = nb;
  L.key = ctx_buf_t<uint64_t>(ctx, s + "key", (size_t)nb);
  L.tb = ctx_buf_t<int>(ctx, s + "tb", (size_t)nb);
  L.te = ctx_buf_t<int>(ctx, s + "te", (size_t)nb);
  L.sb = ctx_buf_t<int>(ctx, s + "sb", (size_t)nb);
  L.se = ctx_buf_t<int>(ctx, s + "se", (size_t)nb);
  L.cb = ctx_buf_t<int>(ctx, s + "cb", (size_t)nb);
  L.ce = ctx_buf_t<int>(ctx, s + "ce", (size_t)nb);
  L.parent = ctx_buf_t<int>(ctx, s + "parent", (size_t)nb);
}

template <typename T>
void build_tree(fmma_ctx* ctx, int d, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src,
                bool lists, int far_from) {
  Tree& tr = ctx->tree;
  tr.valid = false;
  tr.dim = d;
  tr.depth = depth;
  tr.nt = nt;
  tr.ns = ns;
  tr.lev.assign((size_t)depth, Level());
  const int bits = depth - 1;
  const int64_t n = nt + ns;
  const int blk = 256;
  const unsigned g = grid_for(n, blk, (int64_t)ctx->sm_count * 16);

  Cube* cube = compute_cube<T>(ctx, d, nt, tgt, ns, src);
  check_cube(ctx, cube, &tr.cube_host);

  uint64_t* keys = ctx_buf_t<uint64_t>(ctx, "pt_keys", (size_t)n);
  int* idx = ctx_buf_t<int>(ctx, "pt_idx", (size_t)n);
  FMMA_LAUNCH(ctx, (k_leaf_keys<T>), g, blk, 0, tgt, nt, src, ns, d, bits, cube, keys, idx);
  radix_sort_pairs(ctx, keys, idx, n, 0, d * bits);

  int* fbox = ctx_buf_t<int>(ctx, "pt_fbox", (size_t)n);
  int* ft = ctx_buf_t<int>(ctx, "pt_ft", (size_t)n);
  int* boxex = ctx_buf_t<int>(ctx, "pt_boxex", (size_t)n);
  int* tex = ctx_buf_t<int>(ctx, "pt_tex", (size_t)n);
  int* tot = ctx_buf_t<int>(ctx, "tree_tot", 4);
  FMMA_LAUNCH(ctx, k_leaf_flags, g, blk, 0, keys, idx, n, nt, fbox, ft);
  scan_exclusive(ctx, fbox, boxex, n, tot);
  scan_exclusive(ctx, ft, tex, n, tot + 1);
  int hv[2];
  read_ints(ctx, tot, hv, 2);
  const int64_t nleaf = hv[0];

  tr.perm_t = ctx_buf_t<int>(ctx, "perm_t", (size_t)(nt > 0 ? nt : 1));
  tr.perm_s = ctx_buf_t<int>(ctx, "perm_s", (size_t)(ns > 0 ? ns : 1));
  Level& leaf = tr.lev[(size_t)(depth - 1)];
  alloc_level(ctx, leaf, depth - 1, nleaf);
  FMMA_LAUNCH(ctx, k_leaf_emit, g, blk, 0, keys, idx, n, nt, fbox, boxex, tex, tr.perm_t, tr.perm_s,
              leaf.key, leaf.tb, leaf.sb);
  FMMA_LAUNCH(ctx, k_leaf_ends, grid_for(nleaf, blk), blk, 0, nleaf, leaf.tb, leaf.sb, (int)nt,
              (int)ns, leaf.te, leaf.se);
  FMMA_CHECK_CUDA(cudaMemsetAsync(leaf.cb, 0, sizeof(int) * (size_t)nleaf, ctx->stream));
  FMMA_CHECK_CUDA(cudaMemsetAsync(leaf.ce, 0, sizeof(int) * (size_t)nleaf, ctx->stream));

  for (int l = depth - 2; l >= 0; --l) {
    Level& C = tr.lev[(size_t)(l + 1)];
    int* f = ctx_buf_t<int>(ctx, "lv_f", (size_t)C.nbox);
    int* fex = ctx_buf_t<int>(ctx, "lv_fex", (size_t)C.nbox);
    FMMA_LAUNCH(ctx, k_parent_flags, grid_for(C.nbox, blk), blk, 0, C.key, C.nbox, d, f);
    scan_exclusive(ctx, f, fex, C.nbox, tot);
    int np;
    read_ints(ctx, tot, &np, 1);
    Level& Pl = tr.lev[(size_t)l];
    alloc_level(ctx, Pl, l, np);
    FMMA_LAUNCH(ctx, k_parent_emit, grid_for(C.nbox, blk), blk, 0, C.key, C.tb, C.te, C.sb, C.se,
                C.nbox, d, f, fex, C.parent, Pl.key, Pl.tb, Pl.te, Pl.sb, Pl.se, Pl.cb, Pl.ce);
  }
  FMMA_CHECK_CUDA(cudaMemsetAsync(tr.lev[0].parent, 0xff, sizeof(int) * (size_t)tr.lev[0].nbox, ctx->stream));

  if (lists) {
    const FarTables& F = far_tables(d);
    int* slot_j = ctx_buf_t<int>(ctx, "slot_j", 8 * 189);
    FMMA_CHECK_CUDA(cudaMemcpyAsync(slot_j, F.slot_j, sizeof(int) * 8 * 189, cudaMemcpyHostToDevice, ctx->stream));
    unsigned long long* pairs = ctx_buf_t<unsigned long long>(ctx, "il_pairs", depth + 2);
    FMMA_CHECK_CUDA(cudaMemsetAsync(pairs, 0, sizeof(unsigned long long) * (size_t)(depth + 2), ctx->stream));
    for (int l = far_from; l < depth; ++l) {
      Level& Lv = tr.lev[(size_t)l];
      int* f = ctx_buf_t<int>(ctx, "lv_f", (size_t)Lv.nbox);
      int* fex = ctx_buf_t<int>(ctx, "lv_fex", (size_t)Lv.nbox);
      FMMA_LAUNCH(ctx, k_row_flags, grid_for(Lv.nbox, blk), blk, 0, Lv.tb, Lv.te, Lv.nbox, f);
      scan_exclusive(ctx, f, fex, Lv.nbox, tot);
      int nr;
      read_ints(ctx, tot, &nr, 1);
      Lv.nrow = nr;
      std::string s = "lev" + std::to_string(l) + "_";
      uint64_t* ck = ctx_buf_t<uint64_t>(ctx, "row_ck", (size_t)(nr > 0 ? nr : 1));
      Lv.row_box = ctx_buf_t<int>(ctx, s + "row_box", (size_t)(nr > 0 ? nr : 1));
      FMMA_LAUNCH(ctx, k_row_compact, grid_for(Lv.nbox, blk), blk, 0, Lv.key, f, fex, Lv.nbox, d, ck,
                  Lv.row_box);
      radix_sort_pairs(ctx, ck, Lv.row_box, nr, 0, d);
      int* cbd = ctx_buf_t<int>(ctx, "row_cb", 16);
      FMMA_LAUNCH(ctx, k_class_bounds, 1, 32, 0, ck, (int64_t)nr, F.nclass, cbd);
      read_ints(ctx, cbd, Lv.class_begin, F.nclass + 1);
      Lv.il = ctx_buf_t<int>(ctx, s + "il", (size_t)nr * F.nfar + 1);
      if (nr > 0)
        FMMA_LAUNCH(ctx, k_build_il, grid_for((int64_t)nr * F.nfar, blk, (int64_t)ctx->sm_count * 64), blk, 0,
                    Lv.key, Lv.sb, Lv.se, Lv.nbox, Lv.row_box, (int64_t)nr, d, l, F.nfar, slot_j, Lv.il,
                    pairs + l);
    }
    // near lists at the leaf level (rows = leaf boxes with targets, Morton order)
    {
      Level& Lv = tr.lev[(size_t)(depth - 1)];
      int* f = ctx_buf_t<int>(ctx, "lv_f", (size_t)Lv.nbox);
      int* fex = ctx_buf_t<int>(ctx, "lv_fex", (size_t)Lv.nbox);
      FMMA_LAUNCH(ctx, k_row_flags, grid_for(Lv.nbox, blk), blk, 0, Lv.tb, Lv.te, Lv.nbox, f);
      scan_exclusive(ctx, f, fex, Lv.nbox, tot);
      int nr;
      read_ints(ctx, tot, &nr, 1);
      tr.nnear_rows = nr;
      int nnear = d == 1 ? 3 : (d == 2 ? 9 : 27);
      tr.near_row_box = ctx_buf_t<int>(ctx, "near_row_box", (size_t)(nr > 0 ? nr : 1));
      FMMA_LAUNCH(ctx, k_row_compact, grid_for(Lv.nbox, blk), blk, 0, Lv.key, f, fex, Lv.nbox, d,
                  (uint64_t*)nullptr, tr.near_row_box);
      tr.near = ctx_buf_t<int>(ctx, "near", (size_t)nr * nnear + 1);
      if (nr > 0) {
        FMMA_LAUNCH(ctx, k_build_near, grid_for((int64_t)nr * nnear, blk, (int64_t)ctx->sm_count * 64), blk,
                    0, Lv.key, Lv.sb, Lv.se, Lv.nbox, tr.near_row_box, (int64_t)nr, d, depth - 1, nnear,
                    tr.near);
        FMMA_LAUNCH(ctx, k_pairs_p2p, grid_for(nr, blk), blk, 0, tr.near, (int64_t)nr, nnear,
                    tr.near_row_box, Lv.tb, Lv.te, Lv.sb, Lv.se, pairs + depth);
      }
    }
    unsigned long long hp[64];
    unsigned long long* pp = static_cast<unsigned long long*>(ctx_pinned(ctx, sizeof(unsigned long long) * (size_t)(depth + 2)));
    FMMA_CHECK_CUDA(cudaMemcpyAsync(pp, pairs, sizeof(unsigned long long) * (size_t)(depth + 1),
                                    cudaMemcpyDeviceToHost, ctx->stream));
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(hp, pp, sizeof(unsigned long long) * (size_t)(depth + 1));
    for (int l = far_from; l < depth; ++l) tr.lev[(size_t)l].il_pairs = (int64_t)hp[l];
    tr.p2p_pairs = (int64_t)hp[depth];
  }
  tr.valid = true;
}

template void build_tree<double>(fmma_ctx*, int, int, int64_t, const double*, int64_t, const double*, bool, int);
template void build_tree<float>(fmma_ctx*, int, int, int64_t, const float*, int64_t, const float*, bool, int);

// ---------------------------------------------------------------------------
// occupancy and export
// ---------------------------------------------------------------------------
__global__ void k_max_run(const int* __restrict__ tb, const int* __restrict__ te, const int* __restrict__ sb,
                          const int* __restrict__ se, int64_t nb, int* __restrict__ out) {
  int mt = 0, ms = 0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    mt = max(mt, te[b] - tb[b]);
    ms = max(ms, se[b] - sb[b]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mt = max(mt, __shfl_xor_sync(0xffffffffu, mt, o));
    ms = max(ms, __shfl_xor_sync(0xffffffffu, ms, o));
  }
  if ((threadIdx.x & 31) == 0) { atomicMax(out, mt); atomicMax(out + 1, ms); }
}

template <typename T>
void leaf_occupancy(fmma_ctx* ctx, int d, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src,
                    int64_t* max_t, int64_t* max_s) {
  build_tree<T>(ctx, d, depth, nt, tgt, ns, src, false);
  Level& leaf = ctx->tree.lev[(size_t)(depth - 1)];
  int* out = ctx_buf_t<int>(ctx, "occ", 2);
  FMMA_CHECK_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(int), ctx->stream));
  FMMA_LAUNCH(ctx, k_max_run, grid_for(leaf.nbox, 256), 256, 0, leaf.tb, leaf.te, leaf.sb, leaf.se, leaf.nbox, out);
  int h[2];
  read_ints(ctx, out, h, 2);
  *max_t = h[0];
  *max_s = h[1];
  ctx->tree.valid = false;
}

template void leaf_occupancy<double>(fmma_ctx*, int, int, int64_t, const double*, int64_t, const double*, int64_t*, int64_t*);
template void leaf_occupancy<float>(fmma_ctx*, int, int, int64_t, const float*, int64_t, const float*, int64_t*, int64_t*);

__global__ void k_key_to_rowmajor(const uint64_t* __restrict__ keys, int64_t n, int d, int bits,
                                  int64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c[kMaxDim] = {0, 0, 0};
    morton_decode(keys[i], d, bits, c);
    int64_t r = 0;
    for (int q = 0; q < d; ++q) r = (r << bits) | (int64_t)c[q];
    out[i] = r;
  }
}

template <typename T>
void export_bins(fmma_ctx* ctx, int d, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src,
                 int64_t* tbox, int64_t* sbox, Cube* cube_out) {
  Cube* cube = compute_cube<T>(ctx, d, nt, tgt, ns, src);
  check_cube(ctx, cube, cube_out);
  const int64_t n = nt + ns;
  uint64_t* keys = ctx_buf_t<uint64_t>(ctx, "pt_keys", (size_t)(n > 0 ? n : 1));
  const int bits = depth - 1;
  FMMA_LAUNCH(ctx, (k_leaf_keys<T>), grid_for(n, 256), 256, 0, tgt, nt, src, ns, d, bits, cube, keys,
              (int*)nullptr);
  if (nt > 0) FMMA_LAUNCH(ctx, k_key_to_rowmajor, grid_for(nt, 256), 256, 0, keys, nt, d, bits, tbox);
  if (ns > 0) FMMA_LAUNCH(ctx, k_key_to_rowmajor, grid_for(ns, 256), 256, 0, keys + nt, ns, d, bits, sbox);
}

template void export_bins<double>(fmma_ctx*, int, int, int64_t, const double*, int64_t, const double*, int64_t*, int64_t*, Cube*);
template void export_bins<float>(fmma_ctx*, int, int, int64_t, const float*, int64_t, const float*, int64_t*, int64_t*, Cube*);

}  // namespace fmma_b200
