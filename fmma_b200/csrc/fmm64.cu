// fmm64.cu — the plain FP64 FMM on the sparse uniform-depth tree, and the
// exact direct-sum solver.
//
// Stages follow src/fmm.cpp:15-144: P2M at the leaves, M2M up to level 2,
// M2L on levels 2..L-1, L2L down, L2P at the leaves, then P2P over the 3^d
// near leaves.  Operators and interpolation are the reference's
// (src/fmm_core.cpp:222-615, src/math.cpp:14-50).  Coefficient arrays are
// [box][rhs][Kpad] doubles, Kpad = P rounded up to a multiple of 8, pad = 0.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>

#include "fmm_stages.cuh"
#include "fmma_internal.cuh"
#include "kernels.cuh"
#include "m2p.cuh"
#include "solver.cuh"

namespace fmma_b200 {

// ---------------------------------------------------------------------------
// host tables (src/math.cpp:14-50, src/fmm_core.cpp:240-243, :319-336)
// ---------------------------------------------------------------------------
static double host_cheb(int k, double x) { return std::cos(k * std::acos(x)); }
static double host_scheb(int n, double x, double y) {
  double a = 1.0 / n;
  for (int k = 1; k < n; ++k) a += 2.0 / n * host_cheb(k, x) * host_cheb(k, y);
  return a;
}

ChebTables make_cheb_tables(int n) {
  ChebTables t;
  std::memset(&t, 0, sizeof(t));
  t.n = n;
  for (int k = 0; k < n; ++k) t.node[k] = std::cos((2.0 * k + 1.0) / (2 * n) * M_PI);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) t.Tn[k * n + j] = host_cheb(j, t.node[k]);
  for (int s = 0; s < 2; ++s) {
    int shift = 2 * s - 1;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) t.A[s][i * n + j] = host_scheb(n, t.node[i], (t.node[j] + shift) / 2);
  }
  return t;
}

// ---------------------------------------------------------------------------
// point gathers
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_gather_points(const T* __restrict__ p, const int* __restrict__ perm, int64_t n, int d,
                                double* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = perm[i];
    for (int q = 0; q < d; ++q) out[(int64_t)q * n + i] = (double)p[j * d + q];
  }
}

template <typename T>
__global__ void k_gather_weights(const T* __restrict__ w, const int* __restrict__ perm, int64_t ns, int R,
                                 double* __restrict__ out) {
  const int64_t total = ns * R;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e / ns, i = e - r * ns;
    out[e] = w ? (double)w[r * ns + perm[i]] : 1.0;
  }
}

// P2M, M2M, L2L and L2P (forward) run the warp-per-box kernels of fmm_warp.cu.

// ---------------------------------------------------------------------------
// M2L operator tables (src/fmm_core.cpp:383-418), FP64 kernel evaluations:
// tab[f][kl][km] = f(len * x_kl / 2, len * (o_f + x_km / 2)), zero padded
// to [noff][Npad][Kpad].
// ---------------------------------------------------------------------------
template <int KID, int D>
__global__ void k_m2l_table(const double* __restrict__ lens, int ntab, const double* __restrict__ node_all, int P,
                            int Npad, int Kpad, int noff, const int* __restrict__ offv, double p0, int chan,
                            double* __restrict__ tab) {
  const int64_t total = (int64_t)ntab * noff * Npad * Kpad;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t tf = e / ((int64_t)Npad * Kpad);  // table * noff + offset
    const int64_t f = tf % noff;
    const double len = lens[tf / noff];
    int rem = (int)(e - tf * Npad * Kpad);
    int kl = rem / Kpad, km = rem - kl * Kpad;
    double v = 0.0;
    if (kl < P && km < P) {
      double x[D], y[D];
#pragma unroll
      for (int q = 0; q < D; ++q) {
        x[q] = len * (node_all[kl * D + q] / 2);
        y[q] = len * ((double)offv[f * 3 + q] + node_all[km * D + q] / 2);
      }
      if (chan == 0) {
        v = keval<KID, D>(x, y, p0);
      } else {  // derivative channel: d f / d x_{chan-1}
        double g[D];
        kgrad_x<KID, D>(x, y, p0, g);
        v = g[chan - 1];
      }
    }
    tab[e] = v;
  }
}

struct TableLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const double* lens, int ntab, const double* node_all, int P, int Npad, int Kpad,
                  int noff, const int* offv, double p0, int chan, double* tab) {
    int64_t total = (int64_t)ntab * noff * Npad * Kpad;
    FMMA_LAUNCH(ctx, (k_m2l_table<KID, D>), grid_for(total, 256, (int64_t)ctx->sm_count * 32), 256, 0, lens, ntab,
                node_all, P, Npad, Kpad, noff, offv, p0, chan, tab);
  }
};

// ---------------------------------------------------------------------------
// M2L FP64 on the FP64 tensor path (DMMA m8n8k4): a CTA owns 64 target rows
// (box x rhs) of one child-parity class and 32*NBW output coefficients, and
// loops over the class's far slots; per slot the rows gather their source
// box's Wm (K-major) and the slot's operator is the B operand.  3-stage
// cp.async pipeline over (slot, k-chunk of 8).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int kM2LTM = 64, kM2LKC = 8, kM2LST = 3, kM2LLDS = 12;

template <int NBW>
__global__ void __launch_bounds__(256, 1) k_m2l_f64(
    const int4* __restrict__ tiles, const int* __restrict__ il, const int* __restrict__ row_box,
    const int* __restrict__ slot_off, const double* __restrict__ Wm, double* __restrict__ Wl,
    const double* __restrict__ tab, int P, int Kpad, int NpadT, int nfar, int R, int noff) {
  constexpr int TM = kM2LTM, KC = kM2LKC, ST = kM2LST, LDS = kM2LLDS, NW = 32 * NBW;
  extern __shared__ __align__(16) double smem[];
  double* sA = smem;
  double* sB = sA + ST * TM * LDS;
  __shared__ int s_flag[192];
  __shared__ int s_q[192];
  __shared__ int s_nq;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int4 tile = tiles[blockIdx.x];
  const int cls = tile.x, v0 = tile.y, vcnt = tile.z;
  const int ncol0 = blockIdx.y * NW;

  // slots used by at least one row of the tile
  for (int q = tid; q < nfar; q += blockDim.x) s_flag[q] = 0;
  __syncthreads();
  {
    const int b0 = v0 / R, b1 = (v0 + vcnt - 1) / R;
    const int64_t tot = (int64_t)(b1 - b0 + 1) * nfar;
    for (int64_t e = tid; e < tot; e += blockDim.x) {
      int bb = b0 + (int)(e / nfar), q = (int)(e % nfar);
      if (il[(int64_t)bb * nfar + q] >= 0) s_flag[q] = 1;
    }
  }
  __syncthreads();
  if (warp == 0) {
    int base = 0;
    for (int q0 = 0; q0 < nfar; q0 += 32) {
      int q = q0 + lane;
      int f = q < nfar ? s_flag[q] : 0;
      unsigned m = __ballot_sync(0xffffffffu, f);
      if (f) s_q[base + __popc(m & ((1u << lane) - 1u))] = q;
      base += __popc(m);
    }
    if (lane == 0) s_nq = base;
  }
  __syncthreads();
  const int nq = s_nq;
  const int KCH = Kpad / KC;
  const int total = nq * KCH;

  double acc[4][NBW][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < NBW; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // A row owned by this thread for loads
  const int ai = tid >> 2, ap = tid & 3;
  int a_brow = 0, a_r = 0;
  const bool a_ok = ai < vcnt;
  if (a_ok) {
    int v = v0 + ai;
    a_brow = v / R;
    a_r = v - a_brow * R;
  }

  auto load_stage = [&](int it, int st) {
    const int q = s_q[it / KCH];
    const int kc = (it % KCH) * KC;
    const int f = slot_off[cls * 189 + q] + tile.w * noff;
    {
      const double* src = Wm;
      bool ok = false;
      if (a_ok) {
        int s = il[(int64_t)a_brow * nfar + q];
        if (s >= 0) {
          src = Wm + ((int64_t)s * R + a_r) * Kpad + kc + ap * 2;
          ok = true;
        }
      }
      cp_async16(sA + (st * TM + ai) * LDS + ap * 2, src, ok);
    }
    const double* tb = tab + ((int64_t)f * NpadT + ncol0) * Kpad + kc;
    for (int e = tid; e < NW * 4; e += blockDim.x) {
      int nr = e >> 2, p = e & 3;
      cp_async16(sB + (st * NW + nr) * LDS + p * 2, tb + (int64_t)nr * Kpad + p * 2, true);
    }
  };

#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < total) load_stage(s, s);
    cp_async_commit();
  }
  for (int it = 0; it < total; ++it) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    {
      int nx = it + ST - 1;
      if (nx < total) load_stage(nx, nx % ST);
      cp_async_commit();
    }
    const double* A = sA + (it % ST) * TM * LDS;
    const double* B = sB + (it % ST) * NW * LDS;
#pragma unroll
    for (int ks = 0; ks < KC / 4; ++ks) {
      double a[4], b[NBW];
#pragma unroll
      for (int mb = 0; mb < 4; ++mb) a[mb] = A[(wm * 32 + mb * 8 + (lane >> 2)) * LDS + ks * 4 + (lane & 3)];
#pragma unroll
      for (int nb = 0; nb < NBW; ++nb) b[nb] = B[((wn * NBW + nb) * 8 + (lane >> 2)) * LDS + ks * 4 + (lane & 3)];
#pragma unroll
      for (int mb = 0; mb < 4; ++mb)
#pragma unroll
        for (int nb = 0; nb < NBW; ++nb) dmma_m8n8k4(acc[mb][nb][0], acc[mb][nb][1], a[mb], b[nb]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int mb = 0; mb < 4; ++mb) {
    int i = wm * 32 + mb * 8 + (lane >> 2);
    if (i >= vcnt) continue;
    int v = v0 + i;
    int brow = v / R, r = v - brow * R;
    int box = row_box[brow];
    double* dst = Wl + ((int64_t)box * R + r) * Kpad;
#pragma unroll
    for (int nb = 0; nb < NBW; ++nb) {
      int col = ncol0 + (wn * NBW + nb) * 8 + (lane & 3) * 2;
      if (col < P) dst[col] = acc[mb][nb][0];
      if (col + 1 < P) dst[col + 1] = acc[mb][nb][1];
    }
  }
}

template <int NBW>
static void launch_m2l_f64_t(fmma_ctx* ctx, const int4* tiles, int ntiles, int ny, const int* il, const int* row_box,
                             const int* slot_off, const double* Wm, double* Wl, const double* tab, int P, int Kpad,
                             int NpadT, int nfar, int R, int noff) {
  constexpr int NW = 32 * NBW;
  size_t smem = sizeof(double) * (size_t)kM2LST * (kM2LTM + NW) * kM2LLDS;
  static bool attr_set = false;
  if (!attr_set) {
    FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_m2l_f64<NBW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  dim3 grid((unsigned)ntiles, (unsigned)ny);
  FMMA_LAUNCH(ctx, k_m2l_f64<NBW>, grid, 256, smem, tiles, il, row_box, slot_off, Wm, Wl, tab, P, Kpad, NpadT,
              nfar, R, noff);
}

// Columns per CTA for the FP64 M2L: 32*NBW, NBW = ceil(ceil(P/8)/4) capped at 8.
static int m2l_f64_nbw(int P) {
  int nb = (P + 7) / 8;
  int nbw = (nb + 3) / 4;
  return nbw > 8 ? 8 : nbw;
}

static void launch_m2l_f64(fmma_ctx* ctx, const int4* tiles, int ntiles, const int* il, const int* row_box,
                           const int* slot_off, const double* Wm, double* Wl, const double* tab, int P, int Kpad,
                           int NpadT, int nfar, int R, int noff) {
  int nbw = m2l_f64_nbw(P);
  int ny = NpadT / (32 * nbw);
#define FMMA_M2L_CASE(N_) \
  case N_: launch_m2l_f64_t<N_>(ctx, tiles, ntiles, ny, il, row_box, slot_off, Wm, Wl, tab, P, Kpad, NpadT, nfar, R, noff); break;
  switch (nbw) {
    FMMA_M2L_CASE(1) FMMA_M2L_CASE(2) FMMA_M2L_CASE(3) FMMA_M2L_CASE(4)
    FMMA_M2L_CASE(5) FMMA_M2L_CASE(6) FMMA_M2L_CASE(7) default: FMMA_M2L_CASE(8)
  }
#undef FMMA_M2L_CASE
}

// M2L with the operator evaluated per pair on absolute node coordinates
// (src/fmm_core.cpp:456-492): used for kernels that are not translation
// invariant when trans_sym_flag is 0.
template <int KID, int D>
__global__ void k_m2l_pairwise(const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ il, int nfar,
                               const uint64_t* __restrict__ key, int v, const int* __restrict__ depth,
                               const Cube* __restrict__ cubes, const double* __restrict__ node_all, int P, int Kpad,
                               int R, double p0, const double* __restrict__ Wm, double* __restrict__ Wl) {
  for (int64_t row = blockIdx.x; row < nrow; row += gridDim.x) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int l = depth[pid] - 1 - v;
    const double len = c.Len / (double)(1 << l);
    int cl[kMaxDim] = {0, 0, 0};
    morton_decode(key[b] & kMortonMask, D, l, cl);
    for (int kl = threadIdx.x; kl < P; kl += blockDim.x) {
      double x[D];
#pragma unroll
      for (int q = 0; q < D; ++q) x[q] = len * ((double)cl[q] + (1.0 + node_all[kl * D + q]) / 2) + c.origin[q];
      for (int r = 0; r < R; ++r) {
        double acc = 0.0;
        for (int q = 0; q < nfar; ++q) {
          int s = il[row * nfar + q];
          if (s < 0) continue;
          int cm[kMaxDim] = {0, 0, 0};
          morton_decode(key[s] & kMortonMask, D, l, cm);
          const double* w = Wm + ((int64_t)s * R + r) * Kpad;
          for (int km = 0; km < P; ++km) {
            double y[D];
#pragma unroll
            for (int qq = 0; qq < D; ++qq)
              y[qq] = len * ((double)cm[qq] + (1.0 + node_all[km * D + qq]) / 2) + c.origin[qq];
            acc += keval<KID, D>(x, y, p0) * w[km];
          }
        }
        Wl[((int64_t)b * R + r) * Kpad + kl] = acc;
      }
    }
  }
}

struct PairwiseLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const Level& Lv, int nfar, const int* depth, const Cube* cubes,
                  const double* node_all, int P, int Kpad, int R, double p0, const double* Wm, double* Wl) {
    FMMA_LAUNCH(ctx, (k_m2l_pairwise<KID, D>), grid_for(Lv.nrow, 1, (int64_t)ctx->sm_count * 16), 128, 0,
                Lv.row_box, Lv.nrow, Lv.il, nfar, Lv.key, Lv.v, depth, cubes, node_all, P, Kpad, R, p0, Wm, Wl);
  }
};

// ---------------------------------------------------------------------------
// L2P gradient (src/fmm_core.cpp:580-615 differentiated)
// ---------------------------------------------------------------------------
constexpr int kL2PThreads = 128;

// Derivative of the far-field interpolant (the exact derivative of the FMM's
// own L2P, src/fmm_core.cpp:580-615, while the target stays in its leaf):
// potg[r][t][q] = d/dx_q sum_k Wl[k] prod S_n(rel, x_k), d rel/dx = 2/len.
__global__ void __launch_bounds__(kL2PThreads) k_l2p_grad_f64(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ key, const int* __restrict__ tb,
    const int* __restrict__ te, const double* __restrict__ tx, int64_t nt, const Cube* __restrict__ cubes,
    const int* __restrict__ depth, int d, int n, int P, int Kpad, int R, const double* __restrict__ Tn_g,
    const double* __restrict__ Wl, double* __restrict__ pot, double* __restrict__ potg) {
  __shared__ double sTn[kMaxNodes * kMaxNodes];
  extern __shared__ double sW[];
  const int tid = threadIdx.x;
  for (int i = tid; i < n * n; i += blockDim.x) sTn[i] = Tn_g[i];
  const int n0 = n, n1 = d >= 2 ? n : 1, n2 = d >= 3 ? n : 1;
  for (int64_t row = blockIdx.x; row < nrow; row += gridDim.x) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int Nl = 1 << (depth[pid] - 1);
    const double scale = 2.0 * (double)Nl / c.Len;
    __syncthreads();
    for (int i = tid; i < R * Kpad; i += blockDim.x) sW[i] = Wl[(int64_t)b * R * Kpad + i];
    __syncthreads();
    for (int t = tb[b] + tid; t < te[b]; t += blockDim.x) {
      double f[kMaxDim][kMaxNodes], g[kMaxDim][kMaxNodes];
      for (int q = 0; q < kMaxDim; ++q) { f[q][0] = 1.0; g[q][0] = 0.0; }
      for (int q = 0; q < d; ++q)
        cheb_factors_grad(point_rel(tx[(int64_t)q * nt + t], c, q, Nl, false), n, sTn, f[q], g[q]);
      for (int r = 0; r < R; ++r) {
        const double* w = sW + r * Kpad;
        double acc = 0.0, a0 = 0.0, a1 = 0.0, a2 = 0.0;
        int k = 0;
        for (int i0 = 0; i0 < n0; ++i0)
          for (int i1 = 0; i1 < n1; ++i1)
            for (int i2 = 0; i2 < n2; ++i2, ++k) {
              const double f1 = d >= 2 ? f[1][i1] : 1.0, f2 = d >= 3 ? f[2][i2] : 1.0;
              const double wk = w[k];
              acc += wk * f[0][i0] * f1 * f2;
              a0 += wk * g[0][i0] * f1 * f2;
              if (d >= 2) a1 += wk * f[0][i0] * g[1][i1] * f2;
              if (d >= 3) a2 += wk * f[0][i0] * f1 * g[2][i2];
            }
        pot[(int64_t)r * nt + t] = acc;
        double* pg = potg + ((int64_t)r * nt + t) * d;
        pg[0] = a0 * scale;
        if (d >= 2) pg[1] = a1 * scale;
        if (d >= 3) pg[2] = a2 * scale;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// P2P (src/fmm.cpp:121-141): one warp per leaf row; lanes split as
// (target, source subset) and reduce over the subsets with shuffles.
// ---------------------------------------------------------------------------
template <int KID, int D, int RB, typename T>
__global__ void __launch_bounds__(256) k_p2p_f64(
    const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ near, int nnear,
    const int* __restrict__ tb, const int* __restrict__ te, const int* __restrict__ sb, const int* __restrict__ se,
    const double* __restrict__ tx, int64_t nt, const double* __restrict__ sx, int64_t ns,
    const double* __restrict__ ws, int R, double p0, const double* __restrict__ pot,
    const int* __restrict__ perm_t, T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = wid; row < nrow; row += nw) {
    const int b = row_box[row];
    const int t0 = tb[b], t1 = te[b];
    for (int tc = t0; tc < t1; tc += 32) {
      const int cnt = min(32, t1 - tc);
      int tp2 = 1;
      while (tp2 < cnt) tp2 <<= 1;
      const int G = 32 / tp2;
      const int ti = lane & (tp2 - 1), g = lane / tp2;
      const bool tv = ti < cnt;
      double x[D];
#pragma unroll
      for (int q = 0; q < D; ++q) x[q] = tv ? tx[(int64_t)q * nt + tc + ti] : 0.0;
      for (int r0 = 0; r0 < R; r0 += RB) {
        double acc[RB];
#pragma unroll
        for (int r = 0; r < RB; ++r) acc[r] = 0.0;
        if (tv) {
          for (int qn = 0; qn < nnear; ++qn) {
            const int s = near[row * nnear + qn];
            if (s < 0) continue;
            const int j1 = se[s];
            for (int j = sb[s] + g; j < j1; j += G) {
              double y[D];
#pragma unroll
              for (int q = 0; q < D; ++q) y[q] = sx[(int64_t)q * ns + j];
              const double f = keval<KID, D>(x, y, p0);
#pragma unroll
              for (int r = 0; r < RB; ++r)
                if (r0 + r < R) acc[r] += ws[(int64_t)(r0 + r) * ns + j] * f;
            }
          }
        }
#pragma unroll
        for (int r = 0; r < RB; ++r)
          for (int o = tp2; o < 32; o <<= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
        if (g == 0 && tv) {
          const int t = tc + ti;
          const int64_t ot = perm_t[t];
#pragma unroll
          for (int r = 0; r < RB; ++r)
            if (r0 + r < R) {
              double v = acc[r] + (pot ? pot[(int64_t)(r0 + r) * nt + t] : 0.0);
              out[(int64_t)(r0 + r) * nt + ot] = (T)v;
            }
        }
      }
    }
  }
}

template <typename T>
struct P2PLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const Tree& tr, const double* tx, const double* sx, const double* ws, int R,
                  double p0, const double* pot, T* out) {
    const Level& Lf = tr.lev[0];
    const int nnear = D == 1 ? 3 : (D == 2 ? 9 : 27);
    unsigned g = grid_for(tr.nnear_rows * 32, 256, (int64_t)ctx->sm_count * 16);
    if (R == 1)
      FMMA_LAUNCH(ctx, (k_p2p_f64<KID, D, 1, T>), g, 256, 0, tr.near_row_box, tr.nnear_rows, tr.near, nnear, Lf.tb,
                  Lf.te, Lf.sb, Lf.se, tx, tr.nt, sx, tr.ns, ws, R, p0, pot, tr.perm_t, out);
    else
      FMMA_LAUNCH(ctx, (k_p2p_f64<KID, D, 8, T>), g, 256, 0, tr.near_row_box, tr.nnear_rows, tr.near, nnear, Lf.tb,
                  Lf.te, Lf.sb, Lf.se, tx, tr.nt, sx, tr.ns, ws, R, p0, pot, tr.perm_t, out);
  }
};

constexpr int kExactThreads = 256;

// Near field with gradients: out[r][t] = pot + sum w f, grad[r][t][q] =
// potg + sum w d f/d x_q (FP64, warp per leaf row like k_p2p_f64).
template <int KID, int D>
__global__ void __launch_bounds__(256) k_p2p_grad_f64(
    const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ near, int nnear,
    const int* __restrict__ tb, const int* __restrict__ te, const int* __restrict__ sb, const int* __restrict__ se,
    const double* __restrict__ tx, int64_t nt, const double* __restrict__ sx, int64_t ns,
    const double* __restrict__ ws, int R, double p0, const double* __restrict__ pot, const double* __restrict__ potg,
    const int* __restrict__ perm_t, double* __restrict__ out, double* __restrict__ grad) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = wid; row < nrow; row += nw) {
    const int b = row_box[row];
    const int t0 = tb[b], t1 = te[b];
    for (int tc = t0; tc < t1; tc += 32) {
      const int cnt = min(32, t1 - tc);
      int tp2 = 1;
      while (tp2 < cnt) tp2 <<= 1;
      const int G = 32 / tp2;
      const int ti = lane & (tp2 - 1), g = lane / tp2;
      const bool tv = ti < cnt;
      double x[D];
#pragma unroll
      for (int q = 0; q < D; ++q) x[q] = tv ? tx[(int64_t)q * nt + tc + ti] : 0.0;
      for (int r = 0; r < R; ++r) {
        double acc = 0.0, ga[D];
#pragma unroll
        for (int q = 0; q < D; ++q) ga[q] = 0.0;
        if (tv) {
          for (int qn = 0; qn < nnear; ++qn) {
            const int s = near[row * nnear + qn];
            if (s < 0) continue;
            for (int j = sb[s] + g; j < se[s]; j += G) {
              double y[D], gr[D];
#pragma unroll
              for (int q = 0; q < D; ++q) y[q] = sx[(int64_t)q * ns + j];
              const double wj = ws[(int64_t)r * ns + j];
              acc += wj * keval<KID, D>(x, y, p0);
              kgrad_x<KID, D>(x, y, p0, gr);
#pragma unroll
              for (int q = 0; q < D; ++q) ga[q] += wj * gr[q];
            }
          }
        }
        for (int o = tp2; o < 32; o <<= 1) {
          acc += __shfl_xor_sync(0xffffffffu, acc, o);
#pragma unroll
          for (int q = 0; q < D; ++q) ga[q] += __shfl_xor_sync(0xffffffffu, ga[q], o);
        }
        if (g == 0 && tv) {
          const int t = tc + ti;
          const int64_t ot = perm_t[t];
          if (out) out[(int64_t)r * nt + ot] = acc + (pot ? pot[(int64_t)r * nt + t] : 0.0);
#pragma unroll
          for (int q = 0; q < D; ++q)
            grad[((int64_t)r * nt + ot) * D + q] = ga[q] + (potg ? potg[((int64_t)r * nt + t) * D + q] : 0.0);
        }
      }
    }
  }
}

struct P2PGradLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const Tree& tr, const double* tx, const double* sx, const double* ws, int R,
                  double p0, const double* pot, const double* potg, double* out, double* grad) {
    const Level& Lf = tr.lev[0];
    const int nnear = D == 1 ? 3 : (D == 2 ? 9 : 27);
    unsigned g = grid_for(tr.nnear_rows * 32, 256, (int64_t)ctx->sm_count * 16);
    FMMA_LAUNCH(ctx, (k_p2p_grad_f64<KID, D>), g, 256, 0, tr.near_row_box, tr.nnear_rows, tr.near, nnear, Lf.tb, Lf.te,
                Lf.sb, Lf.se, tx, tr.nt, sx, tr.ns, ws, R, p0, pot, potg, tr.perm_t, out, grad);
  }
};

// Exact gradient: grad[r][i][q] = sum_j w[r][j] d f(x_i, y_j) / d x_q.
template <int KID, int D>
__global__ void __launch_bounds__(kExactThreads) k_exact_grad(const double* __restrict__ tgt, int64_t nt,
                                                               const int64_t* __restrict__ rows,
                                                               const double* __restrict__ src, int64_t ns,
                                                               const double* __restrict__ w, int R, double p0,
                                                               double* __restrict__ grad) {
  __shared__ double sy[kExactThreads][D];
  __shared__ double sw[kExactThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < nt;
  const int64_t ti = ok ? (rows ? rows[i] : i) : 0;
  double x[D];
#pragma unroll
  for (int q = 0; q < D; ++q) x[q] = ok ? tgt[ti * D + q] : 0.0;
  for (int r = 0; r < R; ++r) {
    double ga[D];
#pragma unroll
    for (int q = 0; q < D; ++q) ga[q] = 0.0;
    for (int64_t j0 = 0; j0 < ns; j0 += kExactThreads) {
      const int cnt = (int)min((int64_t)kExactThreads, ns - j0);
      __syncthreads();
      if ((int)threadIdx.x < cnt) {
#pragma unroll
        for (int q = 0; q < D; ++q) sy[threadIdx.x][q] = src[(j0 + threadIdx.x) * D + q];
        sw[threadIdx.x] = w ? w[(int64_t)r * ns + j0 + threadIdx.x] : 1.0;
      }
      __syncthreads();
      if (ok)
        for (int j = 0; j < cnt; ++j) {
          double gr[D];
          kgrad_x<KID, D>(x, sy[j], p0, gr);
#pragma unroll
          for (int q = 0; q < D; ++q) ga[q] += sw[j] * gr[q];
        }
    }
    if (ok)
#pragma unroll
      for (int q = 0; q < D; ++q) grad[((int64_t)r * nt + i) * D + q] = ga[q];
  }
}

struct ExactGradLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const double* tgt, int64_t nt, const int64_t* rows, const double* src, int64_t ns,
                  const double* w, int R, double p0, double* grad) {
    FMMA_LAUNCH(ctx, (k_exact_grad<KID, D>), (unsigned)((nt + kExactThreads - 1) / kExactThreads), kExactThreads, 0,
                tgt, nt, rows, src, ns, w, R, p0, grad);
  }
};

void solve_exact_grad(fmma_ctx* ctx, int dim, int64_t nt, const double* tgt, int64_t ns, const double* src, int R,
                      const double* w, double* grad, const int64_t* rows) {
  if (nt == 0) return;
  if (ns == 0) {
    FMMA_CHECK_CUDA(cudaMemsetAsync(grad, 0, sizeof(double) * (size_t)(nt * R * dim), ctx->stream));
    return;
  }
  FMMA_REQUIRE(ctx->kernel_id != kUserKernel, "gradients need a built-in kernel");
  dispatch_kernel<ExactGradLaunch>(ctx->kernel_id, dim, ctx, tgt, nt, rows, src, ns, w, R, ctx->p0, grad);
}

// ---------------------------------------------------------------------------
// exact (src/fmma.cpp:80-101): all pairs, sources staged through shared memory.
// `rows` (optional) restricts the targets to a subset (sampled FP64 oracle).
// ---------------------------------------------------------------------------
template <int KID, int D, typename T>
__global__ void __launch_bounds__(kExactThreads) k_exact(const T* __restrict__ tgt, int64_t nt,
                                                         const int64_t* __restrict__ rows, const T* __restrict__ src,
                                                         int64_t ns, const T* __restrict__ w, int R, double p0,
                                                         T* __restrict__ ans) {
  __shared__ double sy[kExactThreads][D];
  __shared__ double sw[kExactThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < nt;
  const int64_t ti = ok ? (rows ? rows[i] : i) : 0;
  double x[D];
#pragma unroll
  for (int q = 0; q < D; ++q) x[q] = ok ? (double)tgt[ti * D + q] : 0.0;
  for (int r = 0; r < R; ++r) {
    double acc = 0.0;
    for (int64_t j0 = 0; j0 < ns; j0 += kExactThreads) {
      const int cnt = (int)min((int64_t)kExactThreads, ns - j0);
      __syncthreads();
      if ((int)threadIdx.x < cnt) {
#pragma unroll
        for (int q = 0; q < D; ++q) sy[threadIdx.x][q] = (double)src[(j0 + threadIdx.x) * D + q];
        sw[threadIdx.x] = w ? (double)w[(int64_t)r * ns + j0 + threadIdx.x] : 1.0;
      }
      __syncthreads();
      if (ok)
        for (int j = 0; j < cnt; ++j) acc += sw[j] * keval<KID, D>(x, sy[j], p0);
    }
    if (ok) ans[(int64_t)r * nt + i] = (T)acc;
  }
}

template <typename T>
struct ExactLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const T* tgt, int64_t nt, const int64_t* rows, const T* src, int64_t ns, const T* w,
                  int R, double p0, T* ans) {
    FMMA_LAUNCH(ctx, (k_exact<KID, D, T>), (unsigned)((nt + kExactThreads - 1) / kExactThreads), kExactThreads, 0,
                tgt, nt, rows, src, ns, w, R, p0, ans);
  }
};

template <typename T>
void solve_exact(fmma_ctx* ctx, int dim, int64_t nt, const T* tgt, int64_t ns, const T* src, int R, const T* w,
                 T* ans, const int64_t* rows) {
  if (nt == 0) return;
  if (ns == 0) {
    FMMA_CHECK_CUDA(cudaMemsetAsync(ans, 0, sizeof(T) * (size_t)(nt * R), ctx->stream));
    return;
  }
  if (ctx->kernel_id == kUserKernel) {
    fmma_user_launch a{};
    a.what = FMMA_USER_EXACT;
    a.dim = dim;
    a.nrhs = R;
    a.nt = nt;
    a.ns = ns;
    a.tgt = tgt;
    a.src = src;
    a.w = w;
    a.rows = rows;
    a.out = ans;
    a.out_f32 = sizeof(T) == 4;
    call_user_hook(ctx, a);
    return;
  }
  dispatch_kernel<ExactLaunch<T>>(ctx->kernel_id, dim, ctx, tgt, nt, rows, src, ns, w, R, ctx->p0, ans);
}

template void solve_exact<double>(fmma_ctx*, int, int64_t, const double*, int64_t, const double*, int, const double*,
                                  double*, const int64_t*);
template void solve_exact<float>(fmma_ctx*, int, int64_t, const float*, int64_t, const float*, int, const float*,
                                 float*, const int64_t*);

// ---------------------------------------------------------------------------
// operator cache
// ---------------------------------------------------------------------------
double* cached_op(fmma_ctx* ctx, const std::string& key, size_t bytes, bool* fresh) {
  auto it = ctx->ops.find(key);
  if (it != ctx->ops.end()) {
    *fresh = false;
    return static_cast<double*>(it->second.p);
  }
  size_t total = 0;
  for (auto& kv : ctx->ops) total += kv.second.bytes;
  if (total + bytes > (size_t)16 << 30) {  // keep the cache under 16 GiB
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto& kv : ctx->ops) dev_free(ctx, kv.second.p, kv.second.bytes);
    ctx->ops.clear();
  }
  DevBuf b;
  b.p = dev_alloc(ctx, bytes);
  if (!b.p) throw Error(FMMA_ERR_OOM, "operator table allocation of " + std::to_string(bytes) + " bytes failed");
  b.bytes = bytes;
  ctx->ops[key] = b;
  *fresh = true;
  return static_cast<double*>(b.p);
}

std::string op_key(const char* kind, fmma_ctx* ctx, int d, int n, double len, int a, int b) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s_k%d_g%d_p%a_d%d_n%d_len%a_%d_%d", kind, ctx->kernel_id,
                ctx->kernel_id == kUserKernel ? ctx->user_gen : 0, ctx->p0, d, n, len, a, b);
  return buf;
}

// Builds the M2L tile list (class, first virtual row, row count) of a level.
// Tiles of TM rows inside each (problem, class) segment.  Rows of a segment
// are in Morton order, so the i-th of a segment's n tiles covers roughly the
// fraction (i + 1/2) / n of the problem's domain; tiles are listed in that
// order across the classes of a problem, so the tiles that run at the same
// time gather their source rows from one region and share them in L2.
std::vector<int4> m2l_tiles(const Level& Lv, int R, int TM) {
  struct Item {
    int pid;
    double pos;
    int4 t;
  };
  std::vector<Item> items;
  for (const int4& sg : Lv.segs) {  // (problem, class, row_begin, row_end)
    const int tab = Lv.pid_table[(size_t)sg.x];
    const int64_t v0 = (int64_t)sg.z * R, v1 = (int64_t)sg.w * R;
    const int64_t n = (v1 - v0 + TM - 1) / TM;
    int64_t i = 0;
    for (int64_t v = v0; v < v1; v += TM, ++i)
      items.push_back({sg.x, (i + 0.5) / (double)n, make_int4(sg.y, (int)v, (int)std::min<int64_t>(TM, v1 - v), tab)});
  }
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
    return a.pid != b.pid ? a.pid < b.pid : a.pos < b.pos;
  });
  std::vector<int4> t;
  t.reserve(items.size());
  for (const Item& it : items) t.push_back(it.t);
  return t;
}

// Geometry of the FP64 M2L tables.
static void m2l_f64_dims(int P, int* Npad, int* Kpad) {
  *Kpad = (P + 7) / 8 * 8;
  int nw = 32 * m2l_f64_nbw(P);
  *Npad = (P + nw - 1) / nw * nw;
}

// ---------------------------------------------------------------------------
// M2P (src/fmm_core.cpp:624-661), the tree solver's far field: every target
// of a box adds f(x_t, y_k) Wm[s][k] over the Chebyshev nodes y_k of each box
// s on the box's far list at that level.  A block takes one box and a chunk
// of 256 of its targets (blockIdx.y strides over the chunks when the level
// has few boxes); it compacts the box's far list in shared memory (ballot
// prefix, list order kept), then stages batches of far boxes (expansions and
// the 1-D node positions len * (x_o + 1) / 2 + (len * index + origin), as
// the reference forms them) and every thread sweeps the batch for its target
// (m2p.cuh).
// ---------------------------------------------------------------------------
constexpr int kM2PSmem = 40 * 1024;
constexpr int kM2PMaxBatch = 32;
constexpr int kM2PMaxFar = 192;

// TPB threads per block: 256, or 64 on levels whose boxes hold few targets
// (most of a wide block would idle there).
template <int KID, int D, int RB, int TPB>
__global__ void __launch_bounds__(TPB, (RB == 1 ? 768 : 512) / TPB) k_m2p_f64(
    const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ il, int nfar,
    const uint64_t* __restrict__ key, const int* __restrict__ tb, const int* __restrict__ te, int v,
    const int* __restrict__ depth, const Cube* __restrict__ cubes, const double* __restrict__ tx, int64_t nt,
    const double* __restrict__ node_all, int n, int P, int Kpad, int R, int r0, int NB, double p0,
    const double* __restrict__ Wm, double* __restrict__ pot) {
  extern __shared__ double m2p_sm[];
  double* sW = m2p_sm;                        // [NB][RB][P]
  double* sX = sW + (size_t)NB * RB * P;      // [NB][D][n]
  constexpr int kWarps = TPB / 32;
  __shared__ int sList[kM2PMaxFar];
  __shared__ int sWarp[kM2PMaxFar / 32 + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t row = blockIdx.x; row < nrow; row += gridDim.x) {
    const int b = row_box[row];
    const int t0 = tb[b], t1 = te[b];
    if (t0 + (int)blockIdx.y * TPB >= t1) continue;  // block-uniform
    const int pid = key_pid(key[b]);
    const int l = depth[pid] - 1 - v;
    const Cube& c = cubes[pid];
    const double len = c.Len / (double)(1 << l);
    // compact the far list (nfar <= 189), 32-slot groups over the block's warps
    __syncthreads();
    for (int g = warp; g < kM2PMaxFar / 32; g += kWarps) {
      const int i = g * 32 + lane;
      const int sh = i < nfar ? il[row * nfar + i] : -1;
      const unsigned m = __ballot_sync(0xffffffffu, sh >= 0);
      if (lane == 0) sWarp[g] = __popc(m);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int g = 0; g < kM2PMaxFar / 32; ++g) {
        const int cnt = sWarp[g];
        sWarp[g] = acc;
        acc += cnt;
      }
      sWarp[kM2PMaxFar / 32] = acc;
    }
    __syncthreads();
    for (int g = warp; g < kM2PMaxFar / 32; g += kWarps) {
      const int i = g * 32 + lane;
      const int sh = i < nfar ? il[row * nfar + i] : -1;
      const unsigned m = __ballot_sync(0xffffffffu, sh >= 0);
      if (sh >= 0) sList[sWarp[g] + __popc(m & ((1u << lane) - 1u))] = sh;
    }
    const int nlist = sWarp[kM2PMaxFar / 32];
    for (int tc = t0 + (int)blockIdx.y * TPB; tc < t1; tc += (int)gridDim.y * TPB) {
      const int t = tc + (int)threadIdx.x;
      const bool tv = t < t1;
      double x[D];
#pragma unroll
      for (int q = 0; q < D; ++q) x[q] = tv ? tx[(int64_t)q * nt + t] : 0.0;
      double acc[RB];
#pragma unroll
      for (int rr = 0; rr < RB; ++rr) acc[rr] = 0.0;
      for (int bs = 0; bs < nlist; bs += NB) {
        const int nb = min(NB, nlist - bs);
        __syncthreads();
        for (int i = threadIdx.x; i < nb * RB * P; i += blockDim.x) {
          const int j = i / (RB * P), rem = i - j * RB * P, rr = rem / P, k = rem - rr * P;
          sW[i] = r0 + rr < R ? Wm[((int64_t)sList[bs + j] * R + r0 + rr) * Kpad + k] : 0.0;
        }
        for (int i = threadIdx.x; i < nb * D * n; i += blockDim.x) {
          const int j = i / (D * n), rem = i - j * D * n, q = rem / n, o = rem - q * n;
          int cm[kMaxDim] = {0, 0, 0};
          morton_decode(key[sList[bs + j]] & kMortonMask, D, l, cm);
          // node o along dimension q: tensor node (o at digit q, 0 elsewhere)
          int k = o;
          for (int qq = q + 1; qq < D; ++qq) k *= n;
          const double corner = len * (double)cm[q] + c.origin[q];
          sX[i] = (node_all[k * D + q] + 1.0) / 2.0 * len + corner;
        }
        __syncthreads();
        if (tv)
          for (int j = 0; j < nb; ++j) far_box_sum<KID, D, RB>(x, sX + j * D * n, sW + j * RB * P, n, P, p0, acc);
      }
      if (tv) {
#pragma unroll
        for (int rr = 0; rr < RB; ++rr)
          if (r0 + rr < R) pot[(int64_t)(r0 + rr) * nt + t] += acc[rr];
      }
    }
  }
}

template <int KID, int D, int RB, int TPB>
static void m2p_launch(fmma_ctx* ctx, const Level& Lv, int v, int nfar, const int* depth, const Cube* cubes,
                       const double* tx, int64_t nt, const double* node_all, int n, int P, int Kpad, int R, double p0,
                       const double* Wm, double* pot) {
  const int per_box = RB * P * 8 + D * n * 8;
  const int budget = TPB == 256 ? kM2PSmem : kM2PSmem / 4;
  int NB = budget / per_box;
  NB = NB < 1 ? 1 : (NB > kM2PMaxBatch ? kM2PMaxBatch : NB);
  const size_t smem = (size_t)NB * per_box;
  // enough blocks for 4 per SM: split each box's targets over blockIdx.y
  const int64_t gx = std::min<int64_t>(Lv.nrow, (int64_t)ctx->sm_count * 64);
  int64_t gy = ((int64_t)ctx->sm_count * 4 + gx - 1) / gx;
  gy = std::max<int64_t>(1, std::min<int64_t>(gy, 64));
  for (int r0 = 0; r0 < R; r0 += RB)
    FMMA_LAUNCH(ctx, (k_m2p_f64<KID, D, RB, TPB>), dim3((unsigned)gx, (unsigned)gy), TPB, smem, Lv.row_box,
                Lv.nrow, Lv.il, nfar, Lv.key, Lv.tb, Lv.te, v, depth, cubes, tx, nt, node_all, n, P, Kpad, R, r0, NB,
                p0, Wm, pot);
}

template <int KID, int D, int RB>
static void m2p_rb(fmma_ctx* ctx, const Level& Lv, int v, int nfar, const int* depth, const Cube* cubes,
                   const double* tx, int64_t nt, const double* node_all, int n, int P, int Kpad, int R, double p0,
                   const double* Wm, double* pot) {
  // every target lies in one box of each level: nt / rows is the mean occupancy
  if (nt < 128 * Lv.nrow)
    m2p_launch<KID, D, RB, 64>(ctx, Lv, v, nfar, depth, cubes, tx, nt, node_all, n, P, Kpad, R, p0, Wm, pot);
  else
    m2p_launch<KID, D, RB, 256>(ctx, Lv, v, nfar, depth, cubes, tx, nt, node_all, n, P, Kpad, R, p0, Wm, pot);
}

struct M2PLaunch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const Level& Lv, int v, int nfar, const int* depth, const Cube* cubes,
                  const double* tx, int64_t nt, const double* node_all, int n, int P, int Kpad, int R, double p0,
                  const double* Wm, double* pot) {
    if (R == 1) m2p_rb<KID, D, 1>(ctx, Lv, v, nfar, depth, cubes, tx, nt, node_all, n, P, Kpad, R, p0, Wm, pot);
    else if (R <= 4) m2p_rb<KID, D, 4>(ctx, Lv, v, nfar, depth, cubes, tx, nt, node_all, n, P, Kpad, R, p0, Wm, pot);
    else m2p_rb<KID, D, 8>(ctx, Lv, v, nfar, depth, cubes, tx, nt, node_all, n, P, Kpad, R, p0, Wm, pot);
  }
};

// ---------------------------------------------------------------------------
// FP64 near field over the leaves' near lists (src/fmm.cpp:121-141), by the
// built-in kernel or the user hook: out[r][perm_t[t]] = pot[r][t] + sum w f.
// ---------------------------------------------------------------------------
template <typename T>
void near_field_f64(fmma_ctx* ctx, int d, int R, const Tree& tr, const double* tx, const double* sx, const double* ws,
                    const double* pot, T* ans) {
  if (tr.nnear_rows == 0) return;
  if (ctx->kernel_id == kUserKernel) {
    const Level& Lf = tr.lev[0];
    fmma_user_launch ua{};
    ua.what = FMMA_USER_P2P;
    ua.dim = d;
    ua.nrhs = R;
    ua.nrow = tr.nnear_rows;
    ua.row_box = tr.near_row_box;
    ua.near = tr.near;
    ua.nnear = d == 1 ? 3 : (d == 2 ? 9 : 27);
    ua.tb = Lf.tb;
    ua.te = Lf.te;
    ua.sb = Lf.sb;
    ua.se = Lf.se;
    ua.tx = tx;
    ua.nt = tr.nt;
    ua.sx = sx;
    ua.ns = tr.ns;
    ua.ws = ws;
    ua.pot = pot;
    ua.perm_t = tr.perm_t;
    ua.out = ans;
    ua.out_f32 = sizeof(T) == 4;
    call_user_hook(ctx, ua);
  } else {
    dispatch_kernel<P2PLaunch<T>>(ctx->kernel_id, d, ctx, tr, tx, sx, ws, R, ctx->p0, pot, ans);
  }
}

template <typename T>
void launch_gather_points(fmma_ctx* ctx, const T* p, const int* perm, int64_t n, int d, double* out) {
  if (n > 0) FMMA_LAUNCH(ctx, k_gather_points<T>, grid_for(n, 256), 256, 0, p, perm, n, d, out);
}

template <typename T>
void launch_gather_weights(fmma_ctx* ctx, const T* w, const int* perm, int64_t ns, int R, double* out) {
  if (ns > 0) FMMA_LAUNCH(ctx, k_gather_weights<T>, grid_for(ns * R, 256), 256, 0, w, perm, ns, R, out);
}

template void near_field_f64<double>(fmma_ctx*, int, int, const Tree&, const double*, const double*, const double*,
                                     const double*, double*);
template void near_field_f64<float>(fmma_ctx*, int, int, const Tree&, const double*, const double*, const double*,
                                    const double*, float*);
template void launch_gather_points<double>(fmma_ctx*, const double*, const int*, int64_t, int, double*);
template void launch_gather_points<float>(fmma_ctx*, const float*, const int*, int64_t, int, double*);
template void launch_gather_weights<double>(fmma_ctx*, const double*, const int*, int64_t, int, double*);
template void launch_gather_weights<float>(fmma_ctx*, const float*, const int*, int64_t, int, double*);

// ---------------------------------------------------------------------------
// driver: one sweep over a forest (a single solve is a forest of one)
// ---------------------------------------------------------------------------
static uint64_t hash_doubles(const std::vector<double>& v) {
  uint64_t h = 1469598103934665603ull;
  for (double x : v) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof b);
    for (int i = 0; i < 8; ++i) {
      h ^= (b >> (8 * i)) & 0xffu;
      h *= 1099511628211ull;
    }
  }
  return h;
}

template <typename T>
void solve_forest(fmma_ctx* ctx, const SolveArgs& a, const std::vector<int64_t>& toff, const T* tgt,
                  const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth, const T* w, T* ans,
                  double* grad, bool build) {
  const int d = a.dim, n = a.n, P = a.P, R = a.nrhs;
  const int Kpad = (P + 7) / 8 * 8;
  const bool isf = sizeof(T) == 4;

  stage_begin(ctx, ST_TREE);
  if (build) build_forest<T>(ctx, d, toff, tgt, soff, src, depth, true);
  Tree& tr = ctx->tree;
  FMMA_REQUIRE(tr.valid && tr.nprob == (int)depth.size(), "no tree for this sweep");
  const int V = tr.vmax;
  const int64_t nt = tr.nt, ns = tr.ns;
  const Cube* cubes = tr.d_cube;
  const int* ddepth = tr.d_depth;
  double* tx = ctx_buf_t<double>(ctx, "tx", (size_t)(d * nt));
  double* sx = ctx_buf_t<double>(ctx, "sx", (size_t)(d * ns));
  double* ws = ctx_buf_t<double>(ctx, "ws", (size_t)(R * ns));
  if (build) {
    FMMA_LAUNCH(ctx, k_gather_points<T>, grid_for(nt, 256), 256, 0, tgt, tr.perm_t, nt, d, tx);
    FMMA_LAUNCH(ctx, k_gather_points<T>, grid_for(ns, 256), 256, 0, src, tr.perm_s, ns, d, sx);
  }
  // the mixed near field's FP32 weight rows are written by the same gather
  const bool mixed_near =
      !grad && a.precision != FMMA_PREC_FP64 && ctx_translation_invariant(ctx) && ctx->kernel_id != kUserKernel;
  if (mixed_near) gather_weights_mixed<T>(ctx, w, tr.perm_s, ns, R, ws);
  else FMMA_LAUNCH(ctx, k_gather_weights<T>, grid_for(ns * R, 256), 256, 0, w, tr.perm_s, ns, R, ws);
  stage_end(ctx, ST_TREE);

  const double* pot = nullptr;
  const double* potg = nullptr;
  if (V >= 3) {
    ChebTables ct = make_cheb_tables(n);
    double* dTn = ctx_buf_t<double>(ctx, "cheb_Tn", kMaxNodes * kMaxNodes);
    double* dA = ctx_buf_t<double>(ctx, "cheb_A", 2 * kMaxNodes * kMaxNodes);
    std::vector<double> Ap(2 * n * n);
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < n * n; ++i) Ap[s * n * n + i] = ct.A[s][i];
    upload(ctx, dTn, ct.Tn, sizeof(double) * n * n);
    upload(ctx, dA, Ap.data(), sizeof(double) * 2 * n * n);
    std::vector<double> na((size_t)P * d);
    for (int k = 0; k < P; ++k) {
      int kc = k;
      for (int q = d - 1; q >= 0; --q) { na[(size_t)k * d + q] = ct.node[kc % n]; kc /= n; }
    }
    double* node_all = ctx_buf_t<double>(ctx, "node_all", (size_t)P * d);
    upload(ctx, node_all, na.data(), sizeof(double) * P * d);

    // coefficient arrays of every virtual level that some problem uses (real level >= 2)
    std::vector<double*> Wm((size_t)V, nullptr), Wl((size_t)V, nullptr);
    for (int v = 0; v < V; ++v) {
      size_t cnt = (size_t)tr.lev[(size_t)v].nbox * R * Kpad;
      Wm[(size_t)v] = ctx_buf_t<double>(ctx, "Wm" + std::to_string(v), cnt);
      Wl[(size_t)v] = ctx_buf_t<double>(ctx, "Wl" + std::to_string(v), cnt);
    }

    // P2M at the leaves (src/fmm_core.cpp:269-280)
    stage_begin(ctx, ST_P2M);
    {
      const Level& Lf = tr.lev[0];
      launch_p2m_warp(ctx, Lf, sx, ns, ws, R, cubes, ddepth, d, isf, n, P, Kpad, dTn, Wm[0]);
    }
    stage_end(ctx, ST_P2M);

    // M2M up to real level 2 (src/fmm.cpp:62-70)
    stage_begin(ctx, ST_M2M);
    for (int v = 0; v + 1 < V; ++v) {
      const Level& C = tr.lev[(size_t)v];
      const Level& Pl = tr.lev[(size_t)(v + 1)];
      bool any = false;
      for (int p = 0; p < tr.nprob; ++p) any |= tr.depth[(size_t)p] - 1 - (v + 1) >= 2;
      if (!any) break;
      launch_m2m_warp(ctx, C, Pl, v + 1, ddepth, d, n, P, Kpad, R, dA, Wm[(size_t)v], Wm[(size_t)(v + 1)]);
    }
    stage_end(ctx, ST_M2M);

    const FarTables& F = far_tables(d);
    int* slot_off = ctx_buf_t<int>(ctx, "slot_off", 8 * 189);
    int* offv = ctx_buf_t<int>(ctx, "off_vec", 316 * 3);
    upload(ctx, slot_off, F.slot_off, sizeof(int) * 8 * 189);
    upload(ctx, offv, F.off_vec, sizeof(int) * 316 * 3);
    const bool pairwise = !ctx_translation_invariant(ctx) && a.trans_sym != 1;
    const bool user = ctx->kernel_id == kUserKernel;
    if (grad) FMMA_REQUIRE(!pairwise && !user, "gradients need a built-in translation-invariant kernel");
    if (user) FMMA_REQUIRE(tr.nprob == 1, "user kernels run single problems");
    int Npad, Kp;
    m2l_f64_dims(P, &Npad, &Kp);
    double* pt = ctx_buf_t<double>(ctx, "pot", (size_t)(R * nt));
    double* pg = grad ? ctx_buf_t<double>(ctx, "potg", (size_t)(R * nt * d)) : nullptr;
    // leaves of problems with Depth < 3 have no far field
    FMMA_CHECK_CUDA(cudaMemsetAsync(pt, 0, sizeof(double) * (size_t)(R * nt), ctx->stream));
    if (pg) FMMA_CHECK_CUDA(cudaMemsetAsync(pg, 0, sizeof(double) * (size_t)(R * nt * d), ctx->stream));

    if (a.tree) {
      // M2P at every level with rows, into the far-field potential (src/tree.cpp:63-74)
      stage_begin(ctx, ST_M2L);
      for (int v = V - 1; v >= 0; --v) {
        const Level& Lv = tr.lev[(size_t)v];
        if (Lv.nrow == 0) continue;
        dispatch_kernel<M2PLaunch>(ctx->kernel_id, d, ctx, Lv, v, F.nfar, ddepth, cubes, tx, nt, node_all, n, P, Kpad, R,
                                   ctx->p0, Wm[(size_t)v], pt);
      }
      stage_end(ctx, ST_M2L);
    } else {
    // M2L on every level with rows (src/fmm_core.cpp:375-495)
    stage_begin(ctx, ST_M2L);
    for (int v = 0; v < V; ++v) {
      const Level& Lv = tr.lev[(size_t)v];
      if (Lv.nrow == 0) continue;
      if (pairwise) {
        if (user) {
          const int l = tr.depth[0] - 1 - v;
          fmma_user_launch ua{};
          ua.what = FMMA_USER_M2L_PAIRWISE;
          ua.dim = d;
          ua.nrhs = R;
          ua.nrow = Lv.nrow;
          ua.row_box = Lv.row_box;
          ua.il = Lv.il;
          ua.nfar = F.nfar;
          ua.level = l;
          ua.key = Lv.key;
          ua.origin = tr.h_cube[0].origin;
          ua.Len = tr.h_cube[0].Len;
          ua.node_all = node_all;
          ua.P = P;
          ua.kpad = Kpad;
          ua.Wm = Wm[(size_t)v];
          ua.Wl = Wl[(size_t)v];
          call_user_hook(ctx, ua);
        } else {
          dispatch_kernel<PairwiseLaunch>(ctx->kernel_id, d, ctx, Lv, F.nfar, ddepth, cubes, node_all, P, Kpad, R,
                                          ctx->p0, Wm[(size_t)v], Wl[(size_t)v]);
        }
        continue;
      }
      // operator tables, one per problem at this level; the length is the
      // reference's `len` in the caller's type (src/fmm_core.cpp:376)
      const int ntab = (int)Lv.table_pid.size();
      std::vector<double> lens((size_t)ntab);
      for (int t = 0; t < ntab; ++t) {
        const int p = Lv.table_pid[(size_t)t];
        const int l = tr.depth[(size_t)p] - 1 - v;
        const Cube& c = tr.h_cube[(size_t)p];
        lens[(size_t)t] = isf ? (double)(c.Lenf / (float)(1 << l)) : c.Len / (double)(1 << l);
      }
      bool fresh = false;
      const size_t bytes = sizeof(double) * (size_t)ntab * F.noff * Npad * Kp;
      const std::string tkey = op_key("m2l64", ctx, d, n, ntab == 1 ? lens[0] : (double)hash_doubles(lens), Npad, Kp) +
                               "_t" + std::to_string(ntab);
      double* tab = cached_op(ctx, tkey, bytes, &fresh);
      if (fresh) {
        if (user) {
          fmma_user_launch ua{};
          ua.what = FMMA_USER_TABLE;
          ua.dim = d;
          ua.len = lens[0];
          ua.node_all = node_all;
          ua.P = P;
          ua.npad = Npad;
          ua.kpad = Kp;
          ua.noff = F.noff;
          ua.offv = offv;
          ua.tab = tab;
          call_user_hook(ctx, ua);
        } else {
          double* dl = ctx_buf_t<double>(ctx, "table_lens", (size_t)ntab);
          upload(ctx, dl, lens.data(), sizeof(double) * (size_t)ntab);
          dispatch_kernel<TableLaunch>(ctx->kernel_id, d, ctx, dl, ntab, node_all, P, Npad, Kp, F.noff, offv, ctx->p0,
                                       0, tab);
        }
      }
      const int engine = (size_t)v < ctx->m2l_engine.size() ? ctx->m2l_engine[(size_t)v] : -1;
      if (a.precision != FMMA_PREC_FP64 && engine != 0) {
        // engine 1 + 2 i + pair: the 1-SM (pair 0) or 2-SM tensor-core kernel
        // with kM2LUnitChoices[i] units per stage; -1: the context's options
        const int pair = engine > 0 ? (engine - 1) & 1 : -1;
        const int units = engine > 0 ? kM2LUnitChoices[((engine - 1) >> 1) % 3] : -1;
        m2l_level_tc(ctx, a.precision == FMMA_PREC_MIXED_BF16X3, pair, units, Lv, v, F.nfar, slot_off, P, Kpad, R,
                     Wm[(size_t)v], Wl[(size_t)v], tab, Npad, tkey, F.noff, ntab);
        continue;
      }
      std::vector<int4> tiles = m2l_tiles(Lv, R, kM2LTM);
      int4* dt = ctx_buf_t<int4>(ctx, "m2l_tiles" + std::to_string(v), tiles.size());
      upload(ctx, dt, tiles.data(), sizeof(int4) * tiles.size());
      kernel_timer_begin(ctx);
      launch_m2l_f64(ctx, dt, (int)tiles.size(), Lv.il, Lv.row_box, slot_off, Wm[(size_t)v], Wl[(size_t)v], tab, P,
                     Kpad, Npad, F.nfar, R, F.noff);
      kernel_timer_end(ctx, 2.0 * P * P * R, v);
    }
    stage_end(ctx, ST_M2L);

    // L2L top-down into children at real level >= 3 (src/fmm.cpp:99-111); with
    // one right-hand side and sparse leaves the leaf level runs fused into L2P
    const bool fuse_leaf = !grad && R == 1 && V >= 2 && l2lp_leaf_ok(tr.lev[0], nt, d, n, ctx->l2p_mode);
    stage_begin(ctx, ST_L2L);
    for (int v = V - 2; v >= (fuse_leaf ? 1 : 0); --v) {
      const Level& C = tr.lev[(size_t)v];
      if (C.nrow == 0) continue;
      launch_l2l_warp(ctx, C, v, ddepth, d, n, P, Kpad, R, dA, Wl[(size_t)(v + 1)], Wl[(size_t)v]);
    }
    stage_end(ctx, ST_L2L);

    // L2P at the leaves of problems with Depth >= 3 (src/fmm_core.cpp:580-615)
    stage_begin(ctx, ST_L2P);
    {
      const Level& Lf = tr.lev[0];
      const size_t smem_l2p = sizeof(double) * (size_t)R * Kpad;
      FMMA_REQUIRE(smem_l2p <= 200 * 1024, "nrhs * nodes per box too large for L2P");
      if (Lf.nrow > 0) {
        if (grad) {
          if (smem_l2p > 48 * 1024 && !ctx->capturing)
            FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_l2p_grad_f64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem_l2p));
          FMMA_LAUNCH(ctx, k_l2p_grad_f64, grid_for(Lf.nrow, 1, (int64_t)ctx->sm_count * 16), kL2PThreads,
                      smem_l2p, Lf.row_box, Lf.nrow, Lf.key, Lf.tb, Lf.te, tx, nt, cubes, ddepth, d, n, P, Kpad, R,
                      dTn, Wl[0], pt, pg);
        } else if (fuse_leaf) {
          launch_l2lp_leaf(ctx, Lf, tx, nt, cubes, ddepth, d, isf, n, Kpad, dTn, dA, Wl[1], Wl[0], pt);
        } else {
          launch_l2p_warp(ctx, Lf, tx, nt, cubes, ddepth, d, isf, n, P, Kpad, R, dTn, Wl[0], pt, 1, 0);
        }
      }
    }
    stage_end(ctx, ST_L2P);
    }
    pot = pt;
    potg = pg;
  }

  // P2P over the 3^d near leaves (src/fmm.cpp:121-141)
  stage_begin(ctx, ST_P2P);
  if (tr.nnear_rows > 0) {
    if (grad) {
      FMMA_REQUIRE(ctx->kernel_id != kUserKernel, "gradients need a built-in kernel");
      dispatch_kernel<P2PGradLaunch>(ctx->kernel_id, d, ctx, tr, tx, sx, ws, R, ctx->p0, pot, potg, (double*)ans, grad);
    } else if (mixed_near) {
      p2p_mixed<T>(ctx, d, tx, sx, ws, R, pot, ans, true);
    } else {
      near_field_f64<T>(ctx, d, R, tr, tx, sx, ws, pot, ans);
    }
  }
  stage_end(ctx, ST_P2P);
}

template <typename T>
void solve_fmm(fmma_ctx* ctx, const SolveArgs& a, int64_t nt, const T* tgt, int64_t ns, const T* src, const T* w,
               T* ans, double* grad) {
  solve_forest<T>(ctx, a, {0, nt}, tgt, {0, ns}, src, {a.depth}, w, ans, grad, true);
}

template void solve_forest<double>(fmma_ctx*, const SolveArgs&, const std::vector<int64_t>&, const double*,
                                   const std::vector<int64_t>&, const double*, const std::vector<int>&, const double*,
                                   double*, double*, bool);
template void solve_forest<float>(fmma_ctx*, const SolveArgs&, const std::vector<int64_t>&, const float*,
                                  const std::vector<int64_t>&, const float*, const std::vector<int>&, const float*,
                                  float*, double*, bool);
template void solve_fmm<double>(fmma_ctx*, const SolveArgs&, int64_t, const double*, int64_t, const double*,
                                const double*, double*, double*);
template void solve_fmm<float>(fmma_ctx*, const SolveArgs&, int64_t, const float*, int64_t, const float*,
                               const float*, float*, double*);

}  // namespace fmma_b200
