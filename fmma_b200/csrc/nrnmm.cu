// nrnmm.cu — the O(N sqrt N) solver on one uniform grid (src/nrnmm.cpp:13-102).
//
// The bounding cube (src/fmm_core.cpp:158-173) is cut into nrn^d boxes of
// side len = Len / nrn, nrn any positive integer (not a power of two, so the
// Morton tree of the fmm solver does not apply).  Sources are binned and
// expanded in every box (P2M, src/fmm_core.cpp:224-283, the fmm P2M kernel
// run in grid mode).  Each target then takes
//  * the sources of the boxes within one step of its own box in every
//    dimension directly (the fmm near-field kernel over a 3^d near list);
//  * every other box through the box's P Chebyshev nodes weighted by its
//    expansion (M2P, src/nrnmm.cpp:86-97).
// The second part is a dense product of N targets against (boxes x P)
// weighted nodes with a few excluded boxes per target, FP64 compute bound
// (one kernel evaluation and an FMA per pair, m2p.cuh): a block of 256
// consecutive sorted targets stages a batch of boxes (their expansions and
// 1-D node coordinates) in shared memory and every thread sweeps the batch
// for its target, skipping the boxes adjacent to its own.  For small target counts
// the box list is split over blockIdx.y and the partial sums are added in a
// fixed order (deterministic results).
//
// Boxes without sources are skipped in both parts: they add exact zeros,
// where the reference adds f(x, y) * 0 (NaN only when a target sits on a
// node of an empty box).
#include <algorithm>
#include <cmath>
#include <vector>

#include "fmm_stages.cuh"
#include "fmma_internal.cuh"
#include "kernels.cuh"
#include "m2p.cuh"
#include "solver.cuh"

namespace fmma_b200 {

namespace {

// Row-major box number of every point, dimension 0 most significant
// (src/fmm_core.cpp:255-265; targets src/nrnmm.cpp:58-60).
template <typename T>
__global__ void k_grid_keys(const T* __restrict__ p, int64_t n, int d, const Cube* __restrict__ cube, int N,
                            uint64_t* __restrict__ key, int* __restrict__ idx) {
  const Cube c = *cube;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = 0;
    for (int q = 0; q < d; ++q) k = k * (uint64_t)N + (uint64_t)bin_coord<T>(p[i * d + q], c, q, N);
    key[i] = k;
    idx[i] = (int)i;
  }
}

// [b[k], e[k]) = the run of box k in the sorted keys (both zeroed before).
__global__ void k_grid_ranges(const uint64_t* __restrict__ key, int64_t n, int* __restrict__ b, int* __restrict__ e) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = key[i];
    if (i == 0 || key[i - 1] != k) b[k] = (int)i;
    if (i == n - 1 || key[i + 1] != k) e[k] = (int)(i + 1);
  }
}

// Near list of every box: the 3^d boxes at offsets in {-1,0,1}^d (row-major,
// last dimension fastest) that lie in the grid and hold sources, else -1.
__global__ void k_grid_near(int64_t nbox, int d, int N, const int* __restrict__ sb, const int* __restrict__ se,
                            int* __restrict__ row_box, int* __restrict__ near) {
  int p3 = 1;
  for (int q = 0; q < d; ++q) p3 *= 3;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += (int64_t)gridDim.x * blockDim.x) {
    row_box[b] = (int)b;
    int c[kMaxDim] = {0, 0, 0};
    int64_t r = b;
    for (int q = d - 1; q >= 0; --q) { c[q] = (int)(r % N); r /= N; }
    for (int i = 0; i < p3; ++i) {
      int ic = i, ok = 1;
      int64_t s = 0;
      int o[kMaxDim] = {0, 0, 0};
      for (int q = d - 1; q >= 0; --q) { o[q] = ic % 3 - 1; ic /= 3; }
      for (int q = 0; q < d; ++q) {
        const int cq = c[q] + o[q];
        ok &= (cq >= 0 && cq < N) ? 1 : 0;
        s = s * N + cq;
      }
      near[b * p3 + i] = (ok && se[s] > sb[s]) ? (int)s : -1;
    }
  }
}

__global__ void k_grid_flags(int64_t nbox, const int* __restrict__ sb, const int* __restrict__ se,
                             int* __restrict__ flag) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += (int64_t)gridDim.x * blockDim.x)
    flag[b] = se[b] > sb[b] ? 1 : 0;
}

__global__ void k_grid_compact(int64_t nbox, const int* __restrict__ flag, const int* __restrict__ off,
                               int* __restrict__ list) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += (int64_t)gridDim.x * blockDim.x)
    if (flag[b]) list[off[b]] = (int)b;
}

// out[e] = sum_y part[y][e], y in increasing order.
__global__ void k_sum_parts(const double* __restrict__ part, int nsplit, int64_t cnt, double* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int y = 0; y < nsplit; ++y) s += part[(int64_t)y * cnt + e];
    out[e] = s;
  }
}

// ---------------------------------------------------------------------------
// far field (M2P over the whole grid)
// ---------------------------------------------------------------------------
constexpr int kFarThreads = 256;
constexpr int kFarSmem = 40 * 1024;
constexpr int kFarMaxBatch = 32;

__host__ __device__ inline int far_box_bytes(int D, int RB, int P, int n) {
  return RB * P * 8 + D * n * 8 + D * 4;
}

// part[y][r][t] for r in [r0, r0 + RB): the far sum of sorted target t over
// the y-th slice of the source-box list.
template <int KID, int D, int RB>
__global__ void __launch_bounds__(kFarThreads, RB == 1 ? 3 : 2) k_nrn_far(
    const double* __restrict__ tx, int64_t nt, const uint64_t* __restrict__ tkey, const int* __restrict__ sbox,
    const int* __restrict__ nsbox, int N, int n, int P, int Kpad, int R, int r0, int NB,
    const double* __restrict__ gx, const double* __restrict__ Wm, double p0, double* __restrict__ part) {
  extern __shared__ double far_sm[];
  double* sW = far_sm;                                        // [NB][RB][P]
  double* sX = sW + (size_t)NB * RB * P;                      // [NB][D][n]
  int* sB = reinterpret_cast<int*>(sX + (size_t)NB * D * n);  // [NB][D] box coordinates
  const int nsb = *nsbox;
  const int per = (nsb + (int)gridDim.y - 1) / (int)gridDim.y;
  const int b0 = (int)blockIdx.y * per, b1 = min(nsb, b0 + per);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool tv = t < nt;
  double x[D];
  int bi[D];
  {
    uint64_t k = tv ? tkey[t] : 0ull;
#pragma unroll
    for (int q = D - 1; q >= 0; --q) {
      bi[q] = (int)(k % (uint64_t)N);
      k /= (uint64_t)N;
      x[q] = tv ? tx[(int64_t)q * nt + t] : 0.0;
    }
  }
  double acc[RB];
#pragma unroll
  for (int rr = 0; rr < RB; ++rr) acc[rr] = 0.0;
  for (int bs = b0; bs < b1; bs += NB) {
    const int nb = min(NB, b1 - bs);
    __syncthreads();
    for (int i = threadIdx.x; i < nb * RB * P; i += blockDim.x) {
      const int j = i / (RB * P), rem = i - j * RB * P, rr = rem / P, k = rem - rr * P;
      const int s = sbox[bs + j];
      sW[i] = r0 + rr < R ? Wm[((int64_t)s * R + r0 + rr) * Kpad + k] : 0.0;
    }
    for (int i = threadIdx.x; i < nb * D * n; i += blockDim.x) {
      const int j = i / (D * n), rem = i - j * D * n, q = rem / n, o = rem - q * n;
      int s = sbox[bs + j];
      for (int qq = D - 1; qq > q; --qq) s /= N;
      const int dig = s % N;
      sX[i] = gx[((int64_t)q * N + dig) * n + o];
      if (o == 0) sB[j * D + q] = dig;
    }
    __syncthreads();
    if (!tv) continue;
    for (int j = 0; j < nb; ++j) {
      bool near = true;
#pragma unroll
      for (int q = 0; q < D; ++q) near = near && abs(sB[j * D + q] - bi[q]) <= 1;
      if (near) continue;
      far_box_sum<KID, D, RB>(x, sX + j * D * n, sW + j * RB * P, n, P, p0, acc);
    }
  }
  if (tv) {
#pragma unroll
    for (int rr = 0; rr < RB; ++rr)
      if (r0 + rr < R) part[((int64_t)blockIdx.y * R + r0 + rr) * nt + t] = acc[rr];
  }
}

struct FarArgs {
  const double* tx;
  int64_t nt;
  const uint64_t* tkey;
  const int* sbox;
  const int* nsbox;
  int N, n, P, Kpad, R, nsplit;
  const double* gx;
  const double* Wm;
  double* part;
};

template <int KID, int D, int RB>
void far_rb(fmma_ctx* ctx, const FarArgs& f, double p0) {
  const int per_box = far_box_bytes(D, RB, f.P, f.n);
  int NB = kFarSmem / per_box;
  NB = NB < 1 ? 1 : (NB > kFarMaxBatch ? kFarMaxBatch : NB);
  const size_t smem = (size_t)NB * per_box + 16;
  const dim3 grid((unsigned)((f.nt + kFarThreads - 1) / kFarThreads), (unsigned)f.nsplit);
  for (int r0 = 0; r0 < f.R; r0 += RB)
    FMMA_LAUNCH(ctx, (k_nrn_far<KID, D, RB>), grid, kFarThreads, smem, f.tx, f.nt, f.tkey, f.sbox, f.nsbox, f.N, f.n,
                f.P, f.Kpad, f.R, r0, NB, f.gx, f.Wm, p0, f.part);
}

struct FarLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const FarArgs& f, double p0) {
    if (f.R == 1) far_rb<KID, D, 1>(ctx, f, p0);
    else if (f.R <= 4) far_rb<KID, D, 4>(ctx, f, p0);
    else far_rb<KID, D, 8>(ctx, f, p0);
  }
};

// 1-D node coordinates of every grid column, as the reference forms them
// (src/nrnmm.cpp:72-74, :88-90): rel = len * i + origin in the caller's type,
// node position (x_o + 1) / 2 * len + rel in double, stored in the caller's
// type.  Separate statements through volatile keep the host compiler from
// contracting them into FMAs.
template <typename T>
std::vector<double> grid_nodes(const Cube& c, int d, int N, int n);

template <>
std::vector<double> grid_nodes<double>(const Cube& c, int d, int N, int n) {
  std::vector<double> g((size_t)d * N * n);
  const double len = c.Len / N;
  for (int q = 0; q < d; ++q)
    for (int i = 0; i < N; ++i) {
      volatile double m = len * (double)(size_t)i;
      const double rel = m + c.origin[q];
      for (int o = 0; o < n; ++o) {
        const double node = std::cos((2.0 * o + 1.0) / (2 * n) * M_PI);
        volatile double a = (node + 1.0) / 2.0 * len;
        g[((size_t)q * N + i) * n + o] = a + rel;
      }
    }
  return g;
}

template <>
std::vector<double> grid_nodes<float>(const Cube& c, int d, int N, int n) {
  std::vector<double> g((size_t)d * N * n);
  const float len = c.Lenf / N;
  for (int q = 0; q < d; ++q)
    for (int i = 0; i < N; ++i) {
      volatile float m = len * (float)(size_t)i;
      const float rel = m + c.originf[q];
      for (int o = 0; o < n; ++o) {
        const float node = (float)std::cos((2.0 * o + 1.0) / (2 * n) * M_PI);
        volatile double a = ((double)node + 1.0) / 2.0 * (double)len;
        g[((size_t)q * N + i) * n + o] = (double)(float)(a + (double)rel);
      }
    }
  return g;
}

}  // namespace

int nrnmm_default_grid(int64_t ns, int dim, bool isf) {
  const double m = isf ? (double)(float)ns : (double)ns;
  return (int)(std::sqrt(3.0) * std::pow(m, 1.0 / (2.0 * dim))) + 1;
}

template <typename T>
void solve_nrnmm(fmma_ctx* ctx, const SolveArgs& a, int nrn, int64_t nt, const T* tgt, int64_t ns, const T* src,
                 const T* w, T* ans) {
  const int d = a.dim, n = a.n, P = a.P, R = a.nrhs;
  const int Kpad = (P + 7) / 8 * 8;
  const bool isf = sizeof(T) == 4;
  int64_t nbox = 1;
  for (int q = 0; q < d; ++q) nbox *= nrn;
  int bits = 0;
  while (((int64_t)1 << bits) < nbox) ++bits;

  // grid, binning, stable sort by box, box ranges, near lists
  stage_begin(ctx, ST_TREE);
  Cube hc;
  const Cube* dc = problem_cube<T>(ctx, d, nt, tgt, ns, src, "nrn_cube", &hc);
  uint64_t* tkey = ctx_buf_t<uint64_t>(ctx, "nrn_tkey", (size_t)nt);
  uint64_t* skey = ctx_buf_t<uint64_t>(ctx, "nrn_skey", (size_t)ns);
  int* perm_t = ctx_buf_t<int>(ctx, "nrn_perm_t", (size_t)nt);
  int* perm_s = ctx_buf_t<int>(ctx, "nrn_perm_s", (size_t)ns);
  FMMA_LAUNCH(ctx, (k_grid_keys<T>), grid_for(nt, 256), 256, 0, tgt, nt, d, dc, nrn, tkey, perm_t);
  FMMA_LAUNCH(ctx, (k_grid_keys<T>), grid_for(ns, 256), 256, 0, src, ns, d, dc, nrn, skey, perm_s);
  radix_sort_pairs(ctx, tkey, perm_t, nt, 0, bits);
  radix_sort_pairs(ctx, skey, perm_s, ns, 0, bits);

  Tree g;
  g.dim = d;
  g.nt = nt;
  g.ns = ns;
  g.perm_t = perm_t;
  g.perm_s = perm_s;
  g.lev.resize(1);
  Level& L = g.lev[0];
  L.nbox = nbox;
  L.tb = ctx_buf_t<int>(ctx, "nrn_tb", (size_t)nbox);
  L.te = ctx_buf_t<int>(ctx, "nrn_te", (size_t)nbox);
  L.sb = ctx_buf_t<int>(ctx, "nrn_sb", (size_t)nbox);
  L.se = ctx_buf_t<int>(ctx, "nrn_se", (size_t)nbox);
  for (int* p : {L.tb, L.te, L.sb, L.se})
    FMMA_CHECK_CUDA(cudaMemsetAsync(p, 0, sizeof(int) * (size_t)nbox, ctx->stream));
  FMMA_LAUNCH(ctx, k_grid_ranges, grid_for(nt, 256), 256, 0, tkey, nt, L.tb, L.te);
  FMMA_LAUNCH(ctx, k_grid_ranges, grid_for(ns, 256), 256, 0, skey, ns, L.sb, L.se);
  const int p3 = d == 1 ? 3 : (d == 2 ? 9 : 27);
  g.nnear_rows = nbox;
  g.near_row_box = ctx_buf_t<int>(ctx, "nrn_rows", (size_t)nbox);
  g.near = ctx_buf_t<int>(ctx, "nrn_near", (size_t)nbox * p3);
  FMMA_LAUNCH(ctx, k_grid_near, grid_for(nbox, 256), 256, 0, nbox, d, nrn, L.sb, L.se, g.near_row_box, g.near);
  double* tx = ctx_buf_t<double>(ctx, "nrn_tx", (size_t)(d * nt));
  double* sx = ctx_buf_t<double>(ctx, "nrn_sx", (size_t)(d * ns));
  double* ws = ctx_buf_t<double>(ctx, "nrn_ws", (size_t)(R * ns));
  launch_gather_points<T>(ctx, tgt, perm_t, nt, d, tx);
  launch_gather_points<T>(ctx, src, perm_s, ns, d, sx);
  launch_gather_weights<T>(ctx, w, perm_s, ns, R, ws);
  stage_end(ctx, ST_TREE);

  // P2M in every box with sources (src/fmm_core.cpp:269-280)
  stage_begin(ctx, ST_P2M);
  ChebTables ct = make_cheb_tables(n);
  double* dTn = ctx_buf_t<double>(ctx, "nrn_Tn", kMaxNodes * kMaxNodes);
  upload(ctx, dTn, ct.Tn, sizeof(double) * n * n);
  double* Wm = ctx_buf_t<double>(ctx, "nrn_Wm", (size_t)nbox * R * Kpad);
  launch_p2m_warp(ctx, L, sx, ns, ws, R, dc, nullptr, d, isf, n, P, Kpad, dTn, Wm, nrn);
  stage_end(ctx, ST_P2M);

  // M2P from every box that is not adjacent (src/nrnmm.cpp:86-97)
  stage_begin(ctx, ST_M2L);
  double* pot = ctx_buf_t<double>(ctx, "nrn_pot", (size_t)R * nt);
  const std::vector<double> gxh = grid_nodes<T>(hc, d, nrn, n);
  double* gx = ctx_buf_t<double>(ctx, "nrn_gx", gxh.size());
  upload(ctx, gx, gxh.data(), sizeof(double) * gxh.size());
  if (ctx->kernel_id == kUserKernel) {
    fmma_user_launch ua{};
    ua.what = FMMA_USER_NRNMM_FAR;
    ua.dim = d;
    ua.nrhs = R;
    ua.P = P;
    ua.kpad = Kpad;
    ua.nt = nt;
    ua.tx = tx;
    ua.key = tkey;
    ua.sb = L.sb;
    ua.se = L.se;
    ua.Wm = Wm;
    ua.grid_n = nrn;
    ua.n = n;
    ua.gx = gx;
    ua.far = pot;
    call_user_hook(ctx, ua);
  } else {
    int* flag = ctx_buf_t<int>(ctx, "nrn_sflag", (size_t)nbox);
    int* off = ctx_buf_t<int>(ctx, "nrn_soff", (size_t)nbox);
    int* list = ctx_buf_t<int>(ctx, "nrn_slist", (size_t)nbox);
    int* cnt = ctx_buf_t<int>(ctx, "nrn_scount", 1);
    FMMA_LAUNCH(ctx, k_grid_flags, grid_for(nbox, 256), 256, 0, nbox, L.sb, L.se, flag);
    scan_exclusive(ctx, flag, off, nbox, cnt);
    FMMA_LAUNCH(ctx, k_grid_compact, grid_for(nbox, 256), 256, 0, nbox, flag, off, list);
    // enough blocks for every SM: split the box list when the targets alone
    // give fewer than 4 blocks per SM
    const int64_t tblocks = (nt + kFarThreads - 1) / kFarThreads;
    int64_t nsplit = ((int64_t)ctx->sm_count * 4 + tblocks - 1) / tblocks;
    nsplit = std::max<int64_t>(1, std::min<int64_t>({nsplit, nbox / 8 > 0 ? nbox / 8 : 1, 64}));
    double* part = nsplit > 1 ? ctx_buf_t<double>(ctx, "nrn_part", (size_t)nsplit * R * nt) : pot;
    FarArgs f{tx, nt, tkey, list, cnt, nrn, n, P, Kpad, R, (int)nsplit, gx, Wm, part};
    dispatch_kernel<FarLaunch>(ctx->kernel_id, d, ctx, f, ctx->p0);
    if (nsplit > 1)
      FMMA_LAUNCH(ctx, k_sum_parts, grid_for((int64_t)R * nt, 256), 256, 0, part, (int)nsplit, (int64_t)R * nt, pot);
  }
  stage_end(ctx, ST_M2L);

  // sources of the adjacent boxes (src/nrnmm.cpp:78-85)
  stage_begin(ctx, ST_P2P);
  near_field_f64<T>(ctx, d, R, g, tx, sx, ws, pot, ans);
  stage_end(ctx, ST_P2P);
}

template void solve_nrnmm<double>(fmma_ctx*, const SolveArgs&, int, int64_t, const double*, int64_t, const double*,
                                  const double*, double*);
template void solve_nrnmm<float>(fmma_ctx*, const SolveArgs&, int, int64_t, const float*, int64_t, const float*,
                                 const float*, float*);

}  // namespace fmma_b200
