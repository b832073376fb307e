// fmm_warp.cu — warp-per-box kernels for the HBM-bound FMM stages (P2M, L2P,
// M2M, L2L) and the far-list build from parent neighbourhoods.
//
// The stages move a few hundred bytes per point or box and do O(P) flops per
// point, so what limits them is keeping every lane busy and every load
// coalesced, not arithmetic:
//  * P2M (src/fmm_core.cpp:269-280): a warp owns a leaf; lane i owns the
//    coefficients k = i + 32 m.  For each source point, lane q*n + j computes
//    the 1-D factor S_n(x_j, rel_q) (three-term recurrence) and every lane
//    gathers the d factors of its coefficients with shuffles, then adds
//    w_r * prod for a block of right-hand sides held in registers.
//  * L2P (src/fmm_core.cpp:580-615): a warp owns a leaf.  For full leaves
//    lane i owns target i + 32 m, writes its d*n factors to the warp's shared
//    slice and sums Wl[r][k] * prod over k with warp-uniform Wl loads; for
//    sparse leaves lanes own coefficients, as in P2M, and each target's sum
//    is a warp reduction.
//  * M2M / L2L (src/fmm_core.cpp:319-336, :524-541): a warp owns a parent
//    (M2M) or a child (L2L) and applies the separable 1-D operators fibre by
//    fibre in per-warp shared buffers with __syncwarp, so 8 boxes advance per
//    block with no block-wide barrier.
#include "fmm_stages.cuh"
#include "fmma_internal.cuh"

namespace fmma_b200 {

constexpr int kWarpThreads = 256;
constexpr int kWarpsPerBlock = kWarpThreads / 32;

// S_n(node_j, y) = (1 + 2 sum_{m=1}^{n-1} T_m(node_j) T_m(y)) / n (src/math.cpp:32-50),
// evaluated as inv + 2 inv s with inv = 1/n computed once per thread (as
// cheb_factors does): no division on the per-point path.
__device__ __forceinline__ double cheb_factor(const double* sTn, int n, int j, double y, double inv) {
  double t0 = 1.0, t1 = y, s = 0.0;
  for (int m = 1; m < n; ++m) {
    s += sTn[j * n + m] * t1;
    const double t2 = 2.0 * y * t1 - t0;
    t0 = t1;
    t1 = t2;
  }
  return inv + 2.0 * inv * s;
}

// Lane ids of the d factors of coefficient k (last dimension fastest), 5 bits each.
__device__ __forceinline__ int coef_code(int k, int n, int d) {
  int code = 0, kc = k;
  for (int q = d - 1; q >= 0; --q) {
    code |= (q * n + kc % n) << (5 * q);
    kc /= n;
  }
  return code;
}

__device__ __forceinline__ double gather_factors(double f, int code, int d) {
  double p = __shfl_sync(0xffffffffu, f, code & 31);
  if (d >= 2) p *= __shfl_sync(0xffffffffu, f, (code >> 5) & 31);
  if (d >= 3) p *= __shfl_sync(0xffffffffu, f, (code >> 10) & 31);
  return p;
}

// ---------------------------------------------------------------------------
// P2M: Wm[b][r][k] = sum_s w_rs prod_q S_n(x_kq, rel_sq)
// KPL coefficients per lane, RB = 16 / KPL right-hand sides per pass.
// ---------------------------------------------------------------------------
// Several right-hand sides (RB > 1 per pass): the points of a warp's boxes are
// taken in chunks of kP2MChunk: the chunk's
// coordinates X[q][i] and weights W[i][j] (point-major rows of kP2MRow
// doubles) are copied by cp.async into one of two per-warp buffers while the
// previous chunk is summed, the chunk sequence running on across the warp's
// boxes and rhs passes (no per-point global load on the dependent path).
constexpr int kP2MChunk = 32;
constexpr int kP2MMaxPPI = 4;  // points whose factors one warp computes at once (when d * n <= 32 / PPI)
// doubles per staged point: RB rounded up to even (16-byte rows) plus 2, so
// that the lanes' strided writes spread over the banks
template <int RB>
constexpr int kP2MRow = (RB + 1) / 2 * 2 + 2;
template <int RB>
constexpr int kP2MBuf = kMaxDim * kP2MChunk + kP2MChunk * kP2MRow<RB>;  // doubles per buffer

__device__ __forceinline__ void cp_async8_zfill(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}

// One right-hand side: the point loop reads its coordinate and weight from
// global memory directly (loads that do not depend on the previous point's
// sums, so consecutive points' loads overlap); staging in shared memory
// costs more here than it hides.
template <int KPL>
__global__ void __launch_bounds__(kWarpThreads, KPL <= 8 ? 3 : 2) k_p2m_warp1(
    const uint64_t* __restrict__ key, const int* __restrict__ sb, const int* __restrict__ se, int64_t nbox,
    const double* __restrict__ sx, int64_t ns, const double* __restrict__ ws, int R,
    const Cube* __restrict__ cubes, const int* __restrict__ depth, int d, int isf, int n, int P, int Kpad,
    const double* __restrict__ Tn_g, double* __restrict__ Wm, int grid_n) {
  __shared__ double sTn[kMaxNodes * kMaxNodes];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTn[i] = Tn_g[i];
  const double inv_n = 1.0 / n;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int code[KPL];
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    code[i] = k < P ? coef_code(k, n, d) : 0;
  }
  const int fq = lane / n, fj = lane - fq * n;  // the factor this lane computes
  const bool fl = lane < d * n;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t box = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; box < nbox; box += nw) {
    const int s0 = sb[box], s1 = se[box];
    if (s1 <= s0) continue;
    // grid_n > 0: one problem on a uniform grid of grid_n boxes per dimension
    const int pid = grid_n > 0 ? 0 : key_pid(key[box]);
    const Cube& c = cubes[pid];
    const int Nl = grid_n > 0 ? grid_n : 1 << (depth[pid] - 1);
    for (int r = 0; r < R; ++r) {
      double acc[KPL];
#pragma unroll
      for (int i = 0; i < KPL; ++i) acc[i] = 0.0;
      for (int s = s0; s < s1; ++s) {
        double f = 0.0;
        if (fl) f = cheb_factor(sTn, n, fj, point_rel(sx[(int64_t)fq * ns + s], c, fq, Nl, isf != 0), inv_n);
        const double w = ws[(int64_t)r * ns + s];
#pragma unroll
        for (int i = 0; i < KPL; ++i) acc[i] += w * gather_factors(f, code[i], d);
      }
      double* dst = Wm + ((int64_t)box * R + r) * Kpad;
#pragma unroll
      for (int i = 0; i < KPL; ++i) {
        const int k = lane + 32 * i;
        if (k < Kpad) dst[k] = k < P ? acc[i] : 0.0;
      }
    }
  }
}

template <int KPL, int RB>
__global__ void __launch_bounds__(kWarpThreads, 2) k_p2m_warp(
    const uint64_t* __restrict__ key, const int* __restrict__ sb, const int* __restrict__ se, int64_t nbox,
    const double* __restrict__ sx, int64_t ns, const double* __restrict__ ws, int R,
    const Cube* __restrict__ cubes, const int* __restrict__ depth, int d, int isf, int n, int P, int Kpad,
    const double* __restrict__ Tn_g, double* __restrict__ Wm, int grid_n) {
  static_assert(RB > 1, "one right-hand side: k_p2m_warp1");
  constexpr int C = kP2MChunk, ROW = kP2MRow<RB>;
  __shared__ double sTn[kMaxNodes * kMaxNodes];
  extern __shared__ __align__(16) double p2m_buf[];  // per warp: 2 buffers of kP2MBuf<RB> doubles
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTn[i] = Tn_g[i];
  const double inv_n = 1.0 / n;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  double* const wbuf = p2m_buf + (size_t)(threadIdx.x >> 5) * 2 * kP2MBuf<RB>;
  int code[KPL];
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    code[i] = k < P ? coef_code(k, n, d) : 0;
  }
  // ppi points per step: lane pp * d * n + q * n + j computes the factor
  // S_n(x_j, rel_q) of point pp (e.g. 3 points of 10 factors in 2-D with 5
  // nodes), and coefficient codes move by cshift per point
  // (more than 128 coefficients: 3-D with 6 or more nodes, 18 factors, one point)
  constexpr int MAXPPI = KPL <= 4 ? kP2MMaxPPI : 1;
  const int dn = d * n, ppi = min(MAXPPI, 32 / dn);
  const int fpp = lane / dn, fr = lane - fpp * dn, fq = fr / n, fj = fr - fq * n;
  const bool fl = fpp < ppi;
  const int cshift = dn * (1 + (d >= 2 ? 32 : 0) + (d >= 3 ? 1024 : 0));
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;

  // chunk cursor: box, rhs pass r0, chunk start c0, the box's point range [s0, s1)
  struct Cur {
    int64_t box;
    int r0, c0, s0, s1;
  };
  auto next_box = [&](Cur& u, int64_t from) {
    for (int64_t bx = from; bx < nbox; bx += nw) {
      const int a = sb[bx], e = se[bx];
      if (e > a) {
        u = Cur{bx, 0, a, a, e};
        return true;
      }
    }
    return false;
  };
  auto advance = [&](Cur& u) {
    u.c0 += C;
    if (u.c0 < u.s1) return true;
    u.r0 += RB;
    if (u.r0 < R) {
      u.c0 = u.s0;
      return true;
    }
    return next_box(u, u.box + nw);
  };
  auto stage = [&](int b, const Cur& u) {
    const int m = min(C, u.s1 - u.c0);
    double* X = wbuf + (size_t)b * kP2MBuf<RB>;
    double* W = X + kMaxDim * C;
    for (int q = 0; q < d; ++q)
      for (int i = lane; i < m; i += 32) cp_async8_zfill(X + q * C + i, sx + (int64_t)q * ns + u.c0 + i, true);
    // coalesced reads (consecutive points of one rhs), zero beyond R
    for (int j = 0; j < RB; ++j) {
      const bool ok = u.r0 + j < R;
      const double* src = ws + (ok ? (int64_t)(u.r0 + j) * ns + u.c0 : 0);
      for (int i = lane; i < m; i += 32) cp_async8_zfill(W + i * ROW + j, src + (ok ? i : 0), ok);
    }
  };

  Cur cur;
  if (!next_box(cur, ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5)) return;
  stage(0, cur);
  cp_async_commit();
  int buf = 0;
  double acc[RB][KPL];
#pragma unroll
  for (int j = 0; j < RB; ++j)
#pragma unroll
    for (int i = 0; i < KPL; ++i) acc[j][i] = 0.0;
  while (true) {
    Cur nx = cur;
    const bool hn = advance(nx);
    if (hn) stage(buf ^ 1, nx);
    cp_async_commit();
    cp_async_wait<1>();  // this lane's copies of the current chunk have landed
    __syncwarp();        // and every lane's
    // grid_n > 0: one problem on a uniform grid of grid_n boxes per dimension
    const int pid = grid_n > 0 ? 0 : key_pid(key[cur.box]);
    const Cube& c = cubes[pid];
    const int Nl = grid_n > 0 ? grid_n : 1 << (depth[pid] - 1);
    const double* X = wbuf + (size_t)buf * kP2MBuf<RB>;
    const double* W = X + kMaxDim * C;
    const int m = min(C, cur.s1 - cur.c0);
    for (int i = 0; i < m; i += ppi) {
      double f = 0.0;
      if (fl && i + fpp < m) f = cheb_factor(sTn, n, fj, point_rel(X[fq * C + i + fpp], c, fq, Nl, isf != 0), inv_n);
#pragma unroll
      for (int u = 0; u < MAXPPI; ++u) {
        if (u >= ppi || i + u >= m) break;
        double prod[KPL];
#pragma unroll
        for (int k = 0; k < KPL; ++k) prod[k] = gather_factors(f, code[k] + u * cshift, d);
        // the point's RB weights as 16-byte loads
        const double2* wr = reinterpret_cast<const double2*>(W + (i + u) * ROW);
#pragma unroll
        for (int j2 = 0; j2 < (RB + 1) / 2; ++j2) {
          const double2 w2 = wr[j2];
#pragma unroll
          for (int k = 0; k < KPL; ++k) {
            acc[2 * j2][k] += w2.x * prod[k];
            if (2 * j2 + 1 < RB) acc[2 * j2 + 1][k] += w2.y * prod[k];
          }
        }
      }
    }
    __syncwarp();  // buffer buf is restaged two chunks on
    if (!hn || nx.box != cur.box || nx.r0 != cur.r0) {  // the (box, rhs pass) is complete
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (cur.r0 + j < R) {
          double* dst = Wm + ((int64_t)cur.box * R + cur.r0 + j) * Kpad;
#pragma unroll
          for (int k = 0; k < KPL; ++k) {
            const int kk = lane + 32 * k;
            if (kk < Kpad) dst[kk] = kk < P ? acc[j][k] : 0.0;
          }
        }
#pragma unroll
        for (int k = 0; k < KPL; ++k) acc[j][k] = 0.0;
      }
    }
    if (!hn) break;
    cur = nx;
    buf ^= 1;
  }
}

// ---------------------------------------------------------------------------
// L2P: pot[(r * nt + t) * ostride + ooff] = sum_k Wl[leaf][r][k] prod_q S_n(rel_tq, x_kq)
// ---------------------------------------------------------------------------
// Staged row length of k_l2p_warp: every pass reads RB consecutive values
// from r0 (a multiple of RB), so a row holds R rounded up to RB (and to an
// even count), plus 2 doubles of padding.
__host__ __device__ constexpr int l2p_staged_row(int R, int RB) {
  return ((R + RB - 1) / RB * RB + 1) / 2 * 2 + 2;
}

// A leaf's Wl [R][Kpad] copied transposed into dst [Kpad][Rrow] by 8-byte cp.async.
__device__ __forceinline__ void l2p_stage_wl(double* dst, const double* src, int R, int Kpad, int Rrow, int lane) {
  for (int e = lane; e < R * Kpad; e += 32) {
    const int r = e / Kpad, k = e - r * Kpad;
    cp_async8_zfill(dst + k * Rrow + r, src + e, true);
  }
}

// RB right-hand sides per pass (1, 2, 4 or 8, the smallest covering R up to 8).
template <int RB>
__global__ void __launch_bounds__(kWarpThreads, 2) k_l2p_warp(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ key, const int* __restrict__ tb,
    const int* __restrict__ te, const double* __restrict__ tx, int64_t nt, const Cube* __restrict__ cubes,
    const int* __restrict__ depth, int d, int isf, int n, int P, int Kpad, int R, const double* __restrict__ Tn_g,
    const double* __restrict__ Wl, double* __restrict__ pot, int ostride, int ooff, int wl_staged) {
  __shared__ double sTn[kMaxNodes * kMaxNodes];
  // per warp: factors [q*n + j][lane], then (wl_staged) two buffers of a leaf's
  // Wl [Kpad][Rrow]: the next row's is copied (cp.async) while this one is used
  extern __shared__ double sm[];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTn[i] = Tn_g[i];
  const double inv_n = 1.0 / n;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // staged Wl is coefficient-major: row k holds the R values of coefficient k
  // (rows long enough for the last pass's RB values, of an even length plus
  // 2, so that 16-byte loads stay aligned and the transposing writes spread
  // over the banks)
  const int Rrow = l2p_staged_row(R, RB);
  const int wsz = wl_staged ? Rrow * Kpad : 0;
  double* wbase = sm + (size_t)warp * (d * n * 32 + 2 * wsz);
  double* f = wbase + lane;
  double* swl0 = wbase + d * n * 32;
  const int n1 = d >= 2 ? n : 1, n2 = d >= 3 ? n : 1;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int sbuf = 0;
  const int64_t row0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wl_staged && row0 < nrow) l2p_stage_wl(swl0, Wl + (int64_t)row_box[row0] * R * Kpad, R, Kpad, Rrow, lane);
  cp_async_commit();
  for (int64_t row = row0; row < nrow; row += nw) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int Nl = 1 << (depth[pid] - 1);
    const double* wl = Wl + (int64_t)b * R * Kpad;
    double* swl = swl0 + sbuf * wsz;
    if (wl_staged) {
      __syncwarp();  // every lane is done with the buffer restaged now
      if (row + nw < nrow)
        l2p_stage_wl(swl0 + (sbuf ^ 1) * wsz, Wl + (int64_t)row_box[row + nw] * R * Kpad, R, Kpad, Rrow, lane);
      cp_async_commit();
      cp_async_wait<1>();  // this lane's copies of this row have landed
      __syncwarp();        // and every lane's
    }
    for (int t0 = tb[b]; t0 < te[b]; t0 += 32) {
      // a chunk of at most 16 targets with several rhs passes: the two
      // half-warps take the same targets and alternate passes (r0 = 0, RB on
      // the first pass), instead of half the lanes idling through all passes
      int ti = lane, cnt = 32;
      bool split = false;
      if constexpr (RB >= 4) {
        cnt = min(32, te[b] - t0);
        split = cnt <= 16 && R > RB;
        if (split) ti = lane & 15;
      }
      const int t = t0 + ti;
      const bool ok = RB >= 4 ? ti < cnt : t < te[b];
      __syncwarp();
      for (int q = 0; q < d; ++q) {
        const double y = ok ? point_rel(tx[(int64_t)q * nt + t], c, q, Nl, isf != 0) : 0.0;
        for (int j = 0; j < n; ++j) f[(q * n + j) * 32] = cheb_factor(sTn, n, j, y, inv_n);
      }
      __syncwarp();
      for (int r0 = split ? (lane >> 4) * RB : 0; r0 < R; r0 += split ? 2 * RB : RB) {
        double acc[RB];
#pragma unroll
        for (int j = 0; j < RB; ++j) acc[j] = 0.0;
        int k = 0;
        for (int i0 = 0; i0 < n; ++i0) {
          const double a0 = f[i0 * 32];
          for (int i1 = 0; i1 < n1; ++i1) {
            const double a01 = d >= 2 ? a0 * f[(n + i1) * 32] : a0;
            for (int i2 = 0; i2 < n2; ++i2, ++k) {
              const double p = d >= 3 ? a01 * f[(2 * n + i2) * 32] : a01;
              if (wl_staged && RB >= 2) {
                const double2* w2 = reinterpret_cast<const double2*>(swl + k * Rrow + r0);
#pragma unroll
                for (int j2 = 0; j2 < RB / 2; ++j2) {
                  const double2 v = w2[j2];  // entries beyond R are not used
                  acc[2 * j2] += v.x * p;
                  acc[2 * j2 + 1] += v.y * p;
                }
              } else if (wl_staged) {
                acc[0] += swl[k * Rrow + r0] * p;
              } else {
#pragma unroll
                for (int j = 0; j < RB; ++j)
                  if (r0 + j < R) acc[j] += wl[(int64_t)(r0 + j) * Kpad + k] * p;
              }
            }
          }
        }
        if (ok) {
#pragma unroll
          for (int j = 0; j < RB; ++j)
            if (r0 + j < R) pot[((int64_t)(r0 + j) * nt + t) * ostride + ooff] = acc[j];
        }
      }
    }
    sbuf ^= 1;
  }
  cp_async_wait<0>();  // no copy in flight when the warp leaves
}

// L2P with lanes over coefficients (as P2M), for leaves holding few targets:
// per target, factors by lanes, products by shuffles, Wl in registers, one
// warp reduction per right-hand side.
template <int KPL, int RB>
__global__ void __launch_bounds__(kWarpThreads, (RB == 1 && KPL <= 8) ? 3 : 2) k_l2p_coef(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ key, const int* __restrict__ tb,
    const int* __restrict__ te, const double* __restrict__ tx, int64_t nt, const Cube* __restrict__ cubes,
    const int* __restrict__ depth, int d, int isf, int n, int P, int Kpad, int R, const double* __restrict__ Tn_g,
    const double* __restrict__ Wl, double* __restrict__ pot, int ostride, int ooff) {
  __shared__ double sTn[kMaxNodes * kMaxNodes];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sTn[i] = Tn_g[i];
  const double inv_n = 1.0 / n;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int code[KPL];
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    code[i] = k < P ? coef_code(k, n, d) : 0;
  }
  const int fq = lane / n, fj = lane - fq * n;
  const bool fl = lane < d * n;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow; row += nw) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int Nl = 1 << (depth[pid] - 1);
    const int t0 = tb[b], t1 = te[b];
    for (int r0 = 0; r0 < R; r0 += RB) {
      double wl[RB][KPL];
#pragma unroll
      for (int j = 0; j < RB; ++j)
#pragma unroll
        for (int i = 0; i < KPL; ++i) {
          const int k = lane + 32 * i;
          wl[j][i] = (r0 + j < R && k < P) ? Wl[((int64_t)b * R + r0 + j) * Kpad + k] : 0.0;
        }
      for (int t = t0; t < t1; ++t) {
        double f = 0.0;
        if (fl) f = cheb_factor(sTn, n, fj, point_rel(tx[(int64_t)fq * nt + t], c, fq, Nl, isf != 0), inv_n);
        double prod[KPL];
#pragma unroll
        for (int i = 0; i < KPL; ++i) prod[i] = gather_factors(f, code[i], d);
#pragma unroll
        for (int j = 0; j < RB; ++j) {
          if (r0 + j >= R) break;
          double part = 0.0;
#pragma unroll
          for (int i = 0; i < KPL; ++i) part += wl[j][i] * prod[i];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
          if (lane == j) pot[((int64_t)(r0 + j) * nt + t) * ostride + ooff] = part;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// M2M / L2L: separable 1-D operators applied fibre by fibre
// ---------------------------------------------------------------------------
// A warp holds RG right-hand sides of one box (RG * Kpad <= kSepElems
// doubles) in shared memory.  Pass q applies the N x N operator of the box's
// parity along dimension q: lane f takes fibre f (RG * P / N fibres, the N
// coefficients that differ only in digit q), loads it into registers and
// writes its N outputs.  Fibre offsets come from a per-block table, so no
// index arithmetic runs per element.
constexpr int kSepElems = 512;

__device__ __forceinline__ void sep_table(int* tab, int d, int N, int P, int Kpad, int RG) {
  const int nfb = P / N, nf = RG * nfb;
  for (int e = threadIdx.x; e < d * nf; e += blockDim.x) {
    const int q = e / nf, f = e - q * nf;
    const int rr = f / nfb, fi = f - rr * nfb;
    int pw = 1;
    for (int m = q + 1; m < d; ++m) pw *= N;
    tab[e] = rr * Kpad + (fi / pw) * pw * N + fi % pw;
  }
}

// One pass over the warp's fibres: out[off + i pw] = sum_j op(i, j) in[off + j pw],
// op(i, j) = A[i][j] (M2M) or A[j][i] (L2L); ACC adds into `out` instead.
template <int N, bool TRANS, bool ACC>
__device__ __forceinline__ void sep_pass(const double* in, double* out, const double* op, const int* tab, int nfe,
                                         int pw) {
  for (int f = threadIdx.x & 31; f < nfe; f += 32) {
    const int off = tab[f];
    double x[N];
#pragma unroll
    for (int j = 0; j < N; ++j) x[j] = in[off + j * pw];
#pragma unroll 1
    for (int i = 0; i < N; ++i) {
      double y = 0.0;
#pragma unroll
      for (int j = 0; j < N; ++j) y += (TRANS ? op[j * N + i] : op[i * N + j]) * x[j];
      if (ACC) out[off + i * pw] += y; else out[off + i * pw] = y;
    }
  }
}

// The children of a parent in turn: while the passes run on one child's
// expansion (buffer X, scratch Y, sum Z), the next child's is copied by
// cp.async into F (16-byte copies: rows of Kpad doubles, Kpad a multiple of
// 8), so its load latency overlaps the arithmetic; the sums are formed in
// the same order as child by child.  PF false (expansions too large for a
// fourth buffer): each child is loaded when its turn comes.
template <int N, bool PF>
__global__ void __launch_bounds__(kWarpThreads) k_m2m_fib(
    const uint64_t* __restrict__ ckey, const int* __restrict__ csb, const int* __restrict__ cse,
    const uint64_t* __restrict__ pkey, const int* __restrict__ pcb, const int* __restrict__ pce,
    const int* __restrict__ psb, const int* __restrict__ pse, int64_t npar, int vpar,
    const int* __restrict__ depth, int d, int P, int Kpad, int R, int RG, const double* __restrict__ A_g,
    const double* __restrict__ Wc, double* __restrict__ Wp) {
  __shared__ double sA[2 * N * N];
  extern __shared__ double sm[];
  const int nfb = P / N, nf = RG * nfb;
  constexpr int NB = PF ? 4 : 3;
  int* tab = reinterpret_cast<int*>(sm + (size_t)kWarpsPerBlock * NB * RG * Kpad);
  for (int i = threadIdx.x; i < 2 * N * N; i += blockDim.x) sA[i] = A_g[i];
  sep_table(tab, d, N, P, Kpad, RG);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* X = sm + (size_t)warp * NB * RG * Kpad;
  double* Y = X + (size_t)RG * Kpad;
  double* Z = Y + (size_t)RG * Kpad;
  double* F = PF ? Z + (size_t)RG * Kpad : X;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < npar; p += nw) {
    if (pse[p] <= psb[p]) continue;
    if (depth[key_pid(pkey[p])] - 1 - vpar < 2) continue;  // Wm is used on levels >= 2 only
    const int che = pce[p];
    for (int r0 = 0; r0 < R; r0 += RG) {
      const int rg = min(RG, R - r0), ne = rg * Kpad, nfe = rg * nfb;
      for (int e = lane; e < ne; e += 32) Z[e] = 0.0;
      // children holding sources, the first one's copy issued up front
      auto next_child = [&](int c) {
        while (c < che && cse[c] <= csb[c]) ++c;
        return c;
      };
      auto issue = [&](int c, double* dst) {
        const double* src = Wc + ((int64_t)c * R + r0) * Kpad;
        for (int e = 2 * lane; e < ne; e += 64) cp_async16(dst + e, src + e, true);
        cp_async_commit();
      };
      int ch = next_child(pcb[p]);
      if (PF && ch < che) issue(ch, F);
      while (ch < che) {
        const int nx = next_child(ch + 1);
        if (PF) {
          cp_async_wait<0>();  // this lane's copies of child ch have landed
          __syncwarp();
          double* t0 = X;
          X = F;
          F = t0;
          if (nx < che) issue(nx, F);  // F held the previous child, whose passes are done
        } else {
          const double* src = Wc + ((int64_t)ch * R + r0) * Kpad;
          for (int e = lane; e < ne; e += 32) X[e] = src[e];
          __syncwarp();
        }
        const uint64_t kk = ckey[ch];
        const double* in = X;
        double* out = Y;
        int pw = 1;
        for (int q = 1; q < d; ++q) pw *= N;
        for (int q = 0; q < d; ++q, pw /= N) {
          const double* op = sA + (int)((kk >> (d - 1 - q)) & 1ull) * N * N;
          if (q == d - 1) {
            sep_pass<N, false, true>(in, Z, op, tab + q * nf, nfe, pw);
          } else {
            sep_pass<N, false, false>(in, out, op, tab + q * nf, nfe, pw);
            const double* t = in;
            in = out;
            out = const_cast<double*>(t);
          }
          __syncwarp();
        }
        ch = nx;
      }
      double* dst = Wp + ((int64_t)p * R + r0) * Kpad;
      for (int e = lane; e < ne; e += 32) dst[e] = Z[e];
      __syncwarp();
    }
  }
}

// L2L into the rows (boxes with targets) of a level: Wl[b] += op^T Wl[parent(b)].
// CS: register slots a lane holds of the child's expansion block (RG * Kpad
// <= 32 CS doubles); 8 slots keep the kernel at 4 blocks per SM.
template <int N, int CS>
__global__ void __launch_bounds__(kWarpThreads, CS <= 8 ? 4 : 3) k_l2l_fib(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ ckey,
    const int* __restrict__ cparent, int vchild, const int* __restrict__ depth, int d, int P, int Kpad, int R,
    int RG, const double* __restrict__ A_g, const double* __restrict__ Wp, double* __restrict__ Wc) {
  __shared__ double sA[2 * N * N];
  extern __shared__ double sm[];
  const int nfb = P / N, nf = RG * nfb;
  int* tab = reinterpret_cast<int*>(sm + (size_t)kWarpsPerBlock * 2 * RG * Kpad);
  for (int i = threadIdx.x; i < 2 * N * N; i += blockDim.x) sA[i] = A_g[i];
  sep_table(tab, d, N, P, Kpad, RG);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* X = sm + (size_t)warp * 2 * RG * Kpad;
  double* Y = X + (size_t)RG * Kpad;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow; row += nw) {
    const int b = row_box[row];
    const uint64_t kk = ckey[b];
    if (depth[key_pid(kk)] - 1 - vchild < 3) continue;  // the parent has no local expansion
    const int p = cparent[b];
    for (int r0 = 0; r0 < R; r0 += RG) {
      const int rg = min(RG, R - r0), ne = rg * Kpad, nfe = rg * nfb;
      const double* src = Wp + ((int64_t)p * R + r0) * Kpad;
      for (int e = lane; e < ne; e += 32) X[e] = src[e];
      // the child's own expansion (its M2L result), loaded up front into
      // registers: independent loads whose latency overlaps the passes (a
      // load-add-store per element would wait for each load in turn)
      double* dst = Wc + ((int64_t)b * R + r0) * Kpad;
      double cur[CS];
#pragma unroll
      for (int i = 0; i < CS; ++i) {
        const int e = lane + 32 * i;
        cur[i] = e < ne ? dst[e] : 0.0;
      }
      __syncwarp();
      double* in = X;
      double* out = Y;
      int pw = 1;
      for (int q = 1; q < d; ++q) pw *= N;
      for (int q = 0; q < d; ++q, pw /= N) {
        const double* op = sA + (int)((kk >> (d - 1 - q)) & 1ull) * N * N;
        sep_pass<N, true, false>(in, out, op, tab + q * nf, nfe, pw);
        __syncwarp();
        double* t = in;
        in = out;
        out = t;
      }
      // coefficients k < P of each rhs row; the padding stays as it is
#pragma unroll
      for (int i = 0; i < CS; ++i) {
        const int e = lane + 32 * i;
        if (e < ne && e % Kpad < P) dst[e] = cur[i] + in[e];
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// M2M / L2L for small expansions (P <= 32 coefficients: 2-D up to 5 nodes,
// 3-D up to 3): the 2^d child operators M_c = A_{c_0} x ... x A_{c_{d-1}}
// (src/fmm_core.cpp:319-336, :524-541) are built dense in shared memory at
// block start, and a warp applies them with lanes over output coefficients:
// for each input coefficient j one shared-memory operator entry per lane and
// the inputs of up to 16 rhs as warp-uniform 16-byte loads from the warp's
// staged block (coefficient-major), i.e. 16 FMAs per 9 loads, no passes and
// no syncs between dimensions.  The separable kernels above move every
// element through shared memory d times with a __syncwarp per pass, which
// at P = 25 costs more than the 2.5x flops of the dense form saves.
// ---------------------------------------------------------------------------
constexpr int kDenseRB = 16;               // rhs per pass
constexpr int kDenseRow = kDenseRB + 2;    // staged doubles per coefficient (16-byte rows, spread banks)
constexpr int kDenseStage = 32 * kDenseRow;  // per warp

// sM[c][j][i] = M_c[i][j] (M2M: output i, input j) or M_c[j][i] (L2L, the
// transpose), with M_c[a][b] = prod_q A[bit_q(c)][a_q * n + b_q], digits with
// the first dimension slowest and bit_q(c) = bit d-1-q of the child class,
// as the separable passes apply them.
__device__ __forceinline__ void dense_child_ops(double* sM, const double* A_g, int d, int n, int P, bool transpose) {
  const int PP = P * P, total = (1 << d) * PP;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int c = e / PP, rem = e - c * PP, j = rem / P, i = rem - j * P;
    int a = transpose ? j : i, b = transpose ? i : j;
    double m = 1.0;
    for (int q = d - 1; q >= 0; --q) {
      const int bit = (c >> (d - 1 - q)) & 1;
      m *= A_g[bit * n * n + (a % n) * n + (b % n)];
      a /= n;
      b /= n;
    }
    sM[e] = m;
  }
}

// y[r][i] = sum_j sM[c][j][i] x[r][j] for the kDenseRB rhs staged in X
// (X[j * kDenseRow + r]); lane i < P.
__device__ __forceinline__ void dense_apply(const double* M, const double* X, int P, int lane, double* acc) {
  for (int j = 0; j < P; ++j) {
    const double m = lane < P ? M[j * P + lane] : 0.0;
    const double2* xr = reinterpret_cast<const double2*>(X + j * kDenseRow);
#pragma unroll
    for (int r2 = 0; r2 < kDenseRB / 2; ++r2) {
      const double2 v = xr[r2];
      acc[2 * r2] += m * v.x;
      acc[2 * r2 + 1] += m * v.y;
    }
  }
}

// Stage rows src[r * Kpad + j] (r < rg, j < P) into X[j * kDenseRow + r],
// zeros for r >= rg.
__device__ __forceinline__ void dense_stage(double* X, const double* src, int Kpad, int P, int rg, int lane) {
  if (lane < P) {
#pragma unroll
    for (int r = 0; r < kDenseRB; ++r) X[lane * kDenseRow + r] = r < rg ? src[(int64_t)r * Kpad + lane] : 0.0;
  }
}

__global__ void __launch_bounds__(kWarpThreads) k_m2m_dense(
    const uint64_t* __restrict__ ckey, const int* __restrict__ csb, const int* __restrict__ cse,
    const uint64_t* __restrict__ pkey, const int* __restrict__ pcb, const int* __restrict__ pce,
    const int* __restrict__ psb, const int* __restrict__ pse, int64_t npar, int vpar,
    const int* __restrict__ depth, int d, int n, int P, int Kpad, int R, const double* __restrict__ A_g,
    const double* __restrict__ Wc, double* __restrict__ Wp) {
  extern __shared__ __align__(16) double sm[];
  const int nc = 1 << d, PP = P * P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* sM = sm;
  double* X = sm + ((nc * PP + 1) & ~1) + (size_t)warp * kDenseStage;
  dense_child_ops(sM, A_g, d, n, P, false);
  __syncthreads();
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < npar; p += nw) {
    if (pse[p] <= psb[p]) continue;
    if (depth[key_pid(pkey[p])] - 1 - vpar < 2) continue;  // Wm is used on levels >= 2 only
    for (int r0 = 0; r0 < R; r0 += kDenseRB) {
      const int rg = min(kDenseRB, R - r0);
      double acc[kDenseRB];
#pragma unroll
      for (int r = 0; r < kDenseRB; ++r) acc[r] = 0.0;
      for (int ch = pcb[p]; ch < pce[p]; ++ch) {
        if (cse[ch] <= csb[ch]) continue;
        __syncwarp();
        dense_stage(X, Wc + ((int64_t)ch * R + r0) * Kpad, Kpad, P, rg, lane);
        __syncwarp();
        dense_apply(sM + (int)(ckey[ch] & (uint64_t)(nc - 1)) * PP, X, P, lane, acc);
      }
      if (lane < Kpad) {
#pragma unroll
        for (int r = 0; r < kDenseRB; ++r)
          if (r < rg) Wp[((int64_t)p * R + r0 + r) * Kpad + lane] = lane < P ? acc[r] : 0.0;
      }
    }
  }
}

// L2L into the rows of a level, dense form: Wl[b] += M_c^T Wl[parent(b)].
__global__ void __launch_bounds__(kWarpThreads) k_l2l_dense(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ ckey,
    const int* __restrict__ cparent, int vchild, const int* __restrict__ depth, int d, int n, int P, int Kpad, int R,
    const double* __restrict__ A_g, const double* __restrict__ Wp, double* __restrict__ Wc) {
  extern __shared__ __align__(16) double sm[];
  const int nc = 1 << d, PP = P * P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* sM = sm;
  double* X = sm + ((nc * PP + 1) & ~1) + (size_t)warp * kDenseStage;
  dense_child_ops(sM, A_g, d, n, P, true);
  __syncthreads();
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow; row += nw) {
    const int b = row_box[row];
    const uint64_t kk = ckey[b];
    if (depth[key_pid(kk)] - 1 - vchild < 3) continue;  // the parent has no local expansion
    const int p = cparent[b];
    const double* M = sM + (int)(kk & (uint64_t)(nc - 1)) * PP;
    for (int r0 = 0; r0 < R; r0 += kDenseRB) {
      const int rg = min(kDenseRB, R - r0);
      double* dst = Wc + ((int64_t)b * R + r0) * Kpad;
      // the sums start from the child's own expansion (its M2L result),
      // loaded before the staging so that its latency overlaps it
      double acc[kDenseRB];
#pragma unroll
      for (int r = 0; r < kDenseRB; ++r) acc[r] = (r < rg && lane < P) ? dst[(int64_t)r * Kpad + lane] : 0.0;
      __syncwarp();
      dense_stage(X, Wp + ((int64_t)p * R + r0) * Kpad, Kpad, P, rg, lane);
      __syncwarp();
      dense_apply(M, X, P, lane, acc);
      // coefficients k < P of each rhs row; the padding stays as it is
      if (lane < P) {
#pragma unroll
        for (int r = 0; r < kDenseRB; ++r)
          if (r < rg) dst[(int64_t)r * Kpad + lane] = acc[r];
      }
    }
  }
}

// Leaf L2L fused into L2P (one right-hand side, leaves with few targets):
// the leaf's local expansion = its M2L result + the parent's expansion
// translated by the separable L2L passes (src/fmm_core.cpp:524-541), held in
// registers (lanes over coefficients) and evaluated at the leaf's targets as
// k_l2p_coef does (src/fmm_core.cpp:580-615); the leaf expansion is never
// written back.  Leaves at real level < 3 (no parent expansion) use their
// M2L result alone.
template <int N, int D>
__global__ void __launch_bounds__(kWarpThreads, 4) k_l2lp_coef(
    const int* __restrict__ row_box, int64_t nrow, const uint64_t* __restrict__ key, const int* __restrict__ parent,
    const int* __restrict__ tb, const int* __restrict__ te, const double* __restrict__ tx, int64_t nt,
    const Cube* __restrict__ cubes, const int* __restrict__ depth, int isf, int Kpad,
    const double* __restrict__ Tn_g, const double* __restrict__ A_g, const double* __restrict__ Wp,
    const double* __restrict__ Wc, double* __restrict__ pot) {
  constexpr int P = D == 2 ? N * N : N * N * N;
  constexpr int KPL = (P + 31) / 32;
  constexpr int nfb = P / N;
  __shared__ double sTn[N * N];
  __shared__ double sA[2 * N * N];
  __shared__ int tab[D * nfb];
  extern __shared__ double sm_l2lp[];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) sTn[i] = Tn_g[i];
  for (int i = threadIdx.x; i < 2 * N * N; i += blockDim.x) sA[i] = A_g[i];
  sep_table(tab, D, N, P, Kpad, 1);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* X = sm_l2lp + (size_t)warp * 2 * Kpad;
  double* Y = X + Kpad;
  int code[KPL];
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    code[i] = k < P ? coef_code(k, N, D) : 0;
  }
  const int fq = lane / N, fj = lane - fq * N;
  const bool fl = lane < D * N;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow; row += nw) {
    const int b = row_box[row];
    const uint64_t kk = key[b];
    const int pid = key_pid(kk);
    const Cube& c = cubes[pid];
    const int Nl = 1 << (depth[pid] - 1);
    double wl[KPL];
#pragma unroll
    for (int i = 0; i < KPL; ++i) {
      const int k = lane + 32 * i;
      wl[i] = k < P ? Wc[(int64_t)b * Kpad + k] : 0.0;
    }
    if (depth[pid] - 1 >= 3) {  // the parent holds a local expansion
      const double* src = Wp + (int64_t)parent[b] * Kpad;
      for (int e = lane; e < Kpad; e += 32) X[e] = src[e];
      __syncwarp();
      double* in = X;
      double* out = Y;
      int pw = 1;
      for (int q = 1; q < D; ++q) pw *= N;
      for (int q = 0; q < D; ++q, pw /= N) {
        const double* op = sA + (int)((kk >> (D - 1 - q)) & 1ull) * N * N;
        sep_pass<N, true, false>(in, out, op, tab + q * nfb, nfb, pw);
        __syncwarp();
        double* t = in;
        in = out;
        out = t;
      }
#pragma unroll
      for (int i = 0; i < KPL; ++i) {
        const int k = lane + 32 * i;
        if (k < P) wl[i] += in[k];
      }
      __syncwarp();
    }
    for (int t = tb[b]; t < te[b]; ++t) {
      double f = 0.0;
      if (fl) f = cheb_factor(sTn, N, fj, point_rel(tx[(int64_t)fq * nt + t], c, fq, Nl, isf != 0), 1.0 / N);
      double part = 0.0;
#pragma unroll
      for (int i = 0; i < KPL; ++i) part += wl[i] * gather_factors(f, code[i], D);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (lane == 0) pot[t] = part;
    }
  }
}

// ---------------------------------------------------------------------------
// Neighbour and far lists, top-down (src/fmm_core.cpp:15-63, :79-115).  The
// 3^d neighbours of a box (offsets in {-1, 0, 1}^d, the box itself included)
// and its far boxes (the rest of the 6^d window) are all children of its
// parent's neighbours, so each level's lists follow from the level above
// without any key search: one thread per (box, neighbour slot of the parent)
// classifies that neighbour's children by their offset from the box.
// nbr[box][s] = neighbour at offset digits s (last dimension fastest) or -1;
// for rows (row_of_box[box] >= 0) the far children holding sources go to
// il[row][jslot[class][window position]] with their slot_mask bits.  At the
// leaves only boxes holding targets are listed (the near-field rows).  nbr,
// il and slot_mask must be pre-filled (-1, -1, 0).
// ---------------------------------------------------------------------------
__global__ void k_lists_topdown(const uint64_t* __restrict__ key, const int* __restrict__ parent, int64_t nbox,
                                const int* __restrict__ tb, const int* __restrict__ te, bool leaf,
                                const int* __restrict__ sb, const int* __restrict__ se,
                                const int* __restrict__ pnbr, const int* __restrict__ pcb,
                                const int* __restrict__ pce, int d, const int* __restrict__ row_of_box, int nfar,
                                const int* __restrict__ jslot, int* __restrict__ nbr, int* __restrict__ il,
                                unsigned* __restrict__ slot_mask, unsigned long long* __restrict__ pairs) {
  const int nnb = d == 1 ? 3 : (d == 2 ? 9 : 27);
  const int center = (nnb - 1) / 2;
  const int64_t total = nbox * nnb;
  const uint64_t cmask = (1ull << d) - 1ull;
  unsigned long long mine = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e / nnb;
    const int s = (int)(e - b * nnb);
    if (leaf && te[b] <= tb[b]) continue;  // no level below reads a leaf's neighbours: targets only
    const int p = parent[b];
    if (p < 0) {  // a root: its only neighbour is itself
      if (s == center) nbr[b * nnb + center] = (int)b;
      continue;
    }
    const int pn = pnbr[(int64_t)p * nnb + s];
    if (pn < 0) continue;
    const int cls = (int)(key[b] & cmask);
    const int row = row_of_box ? row_of_box[b] : -1;
    int dig[kMaxDim] = {0, 0, 0};
    int sc = s;
    for (int q = d - 1; q >= 0; --q) {
      dig[q] = sc % 3;  // the parent's neighbour at offset dig - 1
      sc /= 3;
    }
    for (int ch = pce[pn] - 1; ch >= pcb[pn]; --ch) {
      const uint64_t ck = key[ch];
      bool near = true;
      int js = 0, jw = 0;
      for (int q = 0; q < d; ++q) {
        const int w = 2 * dig[q] + (int)((ck >> (d - 1 - q)) & 1ull);         // position in the 6^d window
        const int o = w - 2 - (int)((cls >> (d - 1 - q)) & 1);                  // offset from the box
        near = near && o >= -1 && o <= 1;
        js = js * 3 + (o + 1);
        jw = jw * 6 + w;
      }
      if (near) {
        nbr[b * nnb + js] = ch;
      } else if (row >= 0 && se[ch] > sb[ch]) {
        const int slot = jslot[cls * 216 + jw];
        il[(int64_t)row * nfar + slot] = ch;
        atomicOr(slot_mask + (int64_t)row * kSlotWords + (slot >> 5), 1u << (slot & 31));
        ++mine;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(pairs, mine);
}

__global__ void k_rows_of_boxes(const int* __restrict__ row_box, int64_t nrow, int* __restrict__ row_of_box) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrow; r += (int64_t)gridDim.x * blockDim.x)
    row_of_box[row_box[r]] = (int)r;
}

// near[row][s] = the leaf neighbour at slot s when it holds sources, else -1
__global__ void k_near_rows(const int* __restrict__ nbr, const int* __restrict__ row_box, int64_t nrow, int nnb,
                            const int* __restrict__ sb, const int* __restrict__ se, int* __restrict__ near) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nrow * nnb;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / nnb;
    const int s = (int)(e - r * nnb);
    const int nb = nbr[(int64_t)row_box[r] * nnb + s];
    near[e] = (nb >= 0 && se[nb] > sb[nb]) ? nb : -1;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static unsigned warp_grid(fmma_ctx* ctx, int64_t nwork) {
  int64_t g = (nwork + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int64_t cap = (int64_t)ctx->sm_count * 16;
  if (g > cap) g = cap;
  return (unsigned)(g < 1 ? 1 : g);
}

// RB right-hand sides per pass: 1 for a single one, else 16 / KPL (registers)
template <int KPL>
static void p2m_warp_t(fmma_ctx* ctx, const Level& Lf, const double* sx, int64_t ns, const double* ws, int R,
                       const Cube* cubes, const int* depth, int d, bool isf, int n, int P, int Kpad, const double* Tn,
                       double* Wm, int grid_n) {
  constexpr int RBM = KPL >= 16 ? 1 : 16 / KPL;
  if (R == 1 || RBM == 1) {
    FMMA_LAUNCH(ctx, (k_p2m_warp1<KPL>), warp_grid(ctx, Lf.nbox), kWarpThreads, 0, Lf.key, Lf.sb, Lf.se, Lf.nbox, sx,
                ns, ws, R, cubes, depth, d, isf ? 1 : 0, n, P, Kpad, Tn, Wm, grid_n);
  } else if constexpr (RBM > 1) {
    const size_t smem = sizeof(double) * 2 * kP2MBuf<RBM> * kWarpsPerBlock;
    static bool attr = false;
    if (smem > 48 * 1024 && !attr && !ctx->capturing) {
      FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_p2m_warp<KPL, RBM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr = true;
    }
    FMMA_LAUNCH(ctx, (k_p2m_warp<KPL, RBM>), warp_grid(ctx, Lf.nbox), kWarpThreads, smem, Lf.key, Lf.sb, Lf.se,
                Lf.nbox, sx, ns, ws, R, cubes, depth, d, isf ? 1 : 0, n, P, Kpad, Tn, Wm, grid_n);
  }
}

void launch_p2m_warp(fmma_ctx* ctx, const Level& Lf, const double* sx, int64_t ns, const double* ws, int R,
                     const Cube* cubes, const int* depth, int d, bool isf, int n, int P, int Kpad, const double* Tn,
                     double* Wm, int grid_n) {
  FMMA_REQUIRE(d * n <= 32 && Kpad <= 512, "P2M: d * nodes must be <= 32 and P <= 512");
  switch ((Kpad + 31) / 32) {
#define FMMA_P2M_CASE(K_) \
  case K_: p2m_warp_t<K_>(ctx, Lf, sx, ns, ws, R, cubes, depth, d, isf, n, P, Kpad, Tn, Wm, grid_n); break;
    FMMA_P2M_CASE(1) FMMA_P2M_CASE(2) FMMA_P2M_CASE(3) FMMA_P2M_CASE(4) FMMA_P2M_CASE(5) FMMA_P2M_CASE(6)
    FMMA_P2M_CASE(7) FMMA_P2M_CASE(8) FMMA_P2M_CASE(9) FMMA_P2M_CASE(10) FMMA_P2M_CASE(11) FMMA_P2M_CASE(12)
    FMMA_P2M_CASE(13) FMMA_P2M_CASE(14) FMMA_P2M_CASE(15) FMMA_P2M_CASE(16)
#undef FMMA_P2M_CASE
    default: break;
  }
}

void launch_l2p_warp(fmma_ctx* ctx, const Level& Lf, const double* tx, int64_t nt, const Cube* cubes,
                     const int* depth, int d, bool isf, int n, int P, int Kpad, int R, const double* Tn,
                     const double* Wl, double* pot, int ostride, int ooff) {
  FMMA_REQUIRE(d * n <= 32, "L2P: d * nodes must be <= 32");
  // Sparse leaves (a few targets each, as in clustered sets at a uniform
  // depth) leave most lanes of the target-per-lane kernel idle: lanes over
  // coefficients then win.  Full leaves favour lanes over targets.
  if (l2p_coef_lanes(Lf, nt, ctx->l2p_mode)) {
    switch ((Kpad + 31) / 32) {
#define FMMA_L2P_CASE(K_)                                                                                          \
  case K_:                                                                                                        \
    if (R == 1 || K_ >= 16)                                                                                       \
      FMMA_LAUNCH(ctx, (k_l2p_coef<K_, 1>), warp_grid(ctx, Lf.nrow), kWarpThreads, 0, Lf.row_box, Lf.nrow, Lf.key, \
                  Lf.tb, Lf.te, tx, nt, cubes, depth, d, isf ? 1 : 0, n, P, Kpad, R, Tn, Wl, pot, ostride, ooff);    \
    else                                                                                                          \
      FMMA_LAUNCH(ctx, (k_l2p_coef<K_, (K_ >= 16 ? 1 : 16 / K_)>), warp_grid(ctx, Lf.nrow), kWarpThreads, 0,      \
                  Lf.row_box, Lf.nrow, Lf.key, Lf.tb, Lf.te, tx, nt, cubes, depth, d, isf ? 1 : 0, n, P, Kpad, R, Tn, \
                  Wl, pot, ostride, ooff);                                                                        \
    return;
      FMMA_L2P_CASE(1) FMMA_L2P_CASE(2) FMMA_L2P_CASE(3) FMMA_L2P_CASE(4) FMMA_L2P_CASE(5) FMMA_L2P_CASE(6)
      FMMA_L2P_CASE(7) FMMA_L2P_CASE(8) FMMA_L2P_CASE(9) FMMA_L2P_CASE(10) FMMA_L2P_CASE(11) FMMA_L2P_CASE(12)
      FMMA_L2P_CASE(13) FMMA_L2P_CASE(14) FMMA_L2P_CASE(15) FMMA_L2P_CASE(16)
#undef FMMA_L2P_CASE
      default: break;
    }
  }
  const int staged = (int64_t)R * Kpad <= 512 ? 1 : 0;  // the leaf's Wl in shared memory
  const int rb = R >= 8 ? 8 : (R >= 4 ? 4 : (R >= 2 ? 2 : 1));
  const size_t rrow = (size_t)l2p_staged_row(R, rb);  // the kernel's staged row length
  const size_t smem = sizeof(double) * ((size_t)d * n * 32 + (staged ? 2 * rrow * Kpad : 0)) * kWarpsPerBlock;
  switch (rb) {
#define FMMA_L2P_RB(RB_)                                                                                              \
  case RB_:                                                                                                          \
    if (smem > 48 * 1024 && !ctx->capturing)                                                                         \
      FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_l2p_warp<RB_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    FMMA_LAUNCH(ctx, k_l2p_warp<RB_>, warp_grid(ctx, Lf.nrow), kWarpThreads, smem, Lf.row_box, Lf.nrow, Lf.key, Lf.tb,  \
                Lf.te, tx, nt, cubes, depth, d, isf ? 1 : 0, n, P, Kpad, R, Tn, Wl, pot, ostride, ooff, staged);      \
    break;
    FMMA_L2P_RB(1) FMMA_L2P_RB(2) FMMA_L2P_RB(4) FMMA_L2P_RB(8)
#undef FMMA_L2P_RB
    default: break;
  }
}

static int sep_rhs_group(int R, int Kpad) {
  const int g = kSepElems / Kpad;
  return g < 1 ? 1 : (g < R ? g : R);
}

static size_t sep_smem(int nbuf, int d, int n, int P, int Kpad, int RG) {
  return sizeof(double) * (size_t)nbuf * RG * Kpad * kWarpsPerBlock + sizeof(int) * (size_t)d * RG * (P / n);
}

#define FMMA_SEP_CASES(X_) \
  X_(1) X_(2) X_(3) X_(4) X_(5) X_(6) X_(7) X_(8) X_(9) X_(10) X_(11) X_(12) X_(13) X_(14) X_(15) X_(16)

void launch_m2m_warp(fmma_ctx* ctx, const Level& C, const Level& Pl, int vpar, const int* depth, int d, int n, int P,
                     int Kpad, int R, const double* A, const double* Wc, double* Wp) {
  if (P <= 32 && Kpad <= 32) {  // small expansions: dense child operators
    const size_t smem = sizeof(double) * ((((size_t)1 << d) * P * P + 1) / 2 * 2 + (size_t)kWarpsPerBlock * kDenseStage);
    if (smem > 48 * 1024 && !ctx->capturing)
      FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_m2m_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FMMA_LAUNCH(ctx, k_m2m_dense, warp_grid(ctx, Pl.nbox), kWarpThreads, smem, C.key, C.sb, C.se, Pl.key, Pl.cb, Pl.ce,
                Pl.sb, Pl.se, Pl.nbox, vpar, depth, d, n, P, Kpad, R, A, Wc, Wp);
    return;
  }
  const int RG = sep_rhs_group(R, Kpad);
  // X, Y, Z and the prefetch buffer when they fit, else X, Y, Z
  const bool pf = sep_smem(4, d, n, P, Kpad, RG) <= (size_t)160 * 1024;
  const size_t smem = sep_smem(pf ? 4 : 3, d, n, P, Kpad, RG);
  switch (n) {
#define FMMA_M2M_LAUNCH(N_, PF_)                                                                                   \
  if (smem > 48 * 1024 && !ctx->capturing)                                                                        \
    FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_m2m_fib<N_, PF_>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                         (int)smem));                                                            \
  FMMA_LAUNCH(ctx, (k_m2m_fib<N_, PF_>), warp_grid(ctx, Pl.nbox), kWarpThreads, smem, C.key, C.sb, C.se, Pl.key,  \
              Pl.cb, Pl.ce, Pl.sb, Pl.se, Pl.nbox, vpar, depth, d, P, Kpad, R, RG, A, Wc, Wp);
#define FMMA_M2M_CASE(N_)                                                                                          \
  case N_:                                                                                                        \
    if (pf) {                                                                                                     \
      FMMA_M2M_LAUNCH(N_, true)                                                                                   \
    } else {                                                                                                      \
      FMMA_M2M_LAUNCH(N_, false)                                                                                  \
    }                                                                                                             \
    break;
    FMMA_SEP_CASES(FMMA_M2M_CASE)
#undef FMMA_M2M_CASE
#undef FMMA_M2M_LAUNCH
    default: throw Error(FMMA_ERR_INVALID_ARG, "M2M: nodes per dimension must be in [1, 16]");
  }
}

void launch_l2l_warp(fmma_ctx* ctx, const Level& C, int vchild, const int* depth, int d, int n, int P, int Kpad, int R,
                     const double* A, const double* Wp, double* Wc) {
  if (P <= 32 && Kpad <= 32) {  // small expansions: dense child operators
    const size_t smem = sizeof(double) * ((((size_t)1 << d) * P * P + 1) / 2 * 2 + (size_t)kWarpsPerBlock * kDenseStage);
    if (smem > 48 * 1024 && !ctx->capturing)
      FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_l2l_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FMMA_LAUNCH(ctx, k_l2l_dense, warp_grid(ctx, C.nrow), kWarpThreads, smem, C.row_box, C.nrow, C.key, C.parent,
                vchild, depth, d, n, P, Kpad, R, A, Wp, Wc);
    return;
  }
  const int RG = sep_rhs_group(R, Kpad);
  const size_t smem = sep_smem(2, d, n, P, Kpad, RG);
  const bool wide = RG * Kpad > 256;  // 16 register slots a lane, else 8
  switch (n) {
#define FMMA_L2L_LAUNCH(N_, CS_)                                                                                   \
  {                                                                                                               \
    if (smem > 48 * 1024 && !ctx->capturing)                                                                      \
      FMMA_CHECK_CUDA(                                                                                            \
          cudaFuncSetAttribute(k_l2l_fib<N_, CS_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));      \
    FMMA_LAUNCH(ctx, (k_l2l_fib<N_, CS_>), warp_grid(ctx, C.nrow), kWarpThreads, smem, C.row_box, C.nrow, C.key,  \
                C.parent, vchild, depth, d, P, Kpad, R, RG, A, Wp, Wc);                                          \
  }
#define FMMA_L2L_CASE(N_)                      \
  case N_:                                     \
    if (wide) FMMA_L2L_LAUNCH(N_, 16)          \
    else FMMA_L2L_LAUNCH(N_, 8)                \
    break;
    FMMA_SEP_CASES(FMMA_L2L_CASE)
#undef FMMA_L2L_CASE
#undef FMMA_L2L_LAUNCH
    default: throw Error(FMMA_ERR_INVALID_ARG, "L2L: nodes per dimension must be in [1, 16]");
  }
}

// Lanes over coefficients for the leaves: forced by mode 2, refused by mode 1,
// else when the leaves hold fewer than 16 targets on average.
bool l2p_coef_lanes(const Level& Lf, int64_t nt, int mode) {
  return mode == 2 || (mode == 0 && nt < 16 * Lf.nrow);
}

bool l2lp_leaf_ok(const Level& Lf, int64_t nt, int d, int n, int mode) {
  if (Lf.nrow == 0 || !l2p_coef_lanes(Lf, nt, mode)) return false;  // dense leaves: the target-lane L2P
  return (d == 3 && n >= 4 && n <= 7) || (d == 2 && n >= 4 && n <= 8);
}

bool launch_l2lp_leaf(fmma_ctx* ctx, const Level& Lf, const double* tx, int64_t nt, const Cube* cubes,
                      const int* depth, int d, bool isf, int n, int Kpad, const double* Tn, const double* A,
                      const double* Wp, const double* Wc, double* pot) {
  if (!l2lp_leaf_ok(Lf, nt, d, n, ctx->l2p_mode)) return false;
  const size_t smem = sizeof(double) * (size_t)2 * Kpad * kWarpsPerBlock;
#define FMMA_L2LP_CASE(N_, D_)                                                                                    \
  if (n == N_ && d == D_) {                                                                                       \
    FMMA_LAUNCH(ctx, (k_l2lp_coef<N_, D_>), warp_grid(ctx, Lf.nrow), kWarpThreads, smem, Lf.row_box, Lf.nrow,    \
                Lf.key, Lf.parent, Lf.tb, Lf.te, tx, nt, cubes, depth, isf ? 1 : 0, Kpad, Tn, A, Wp, Wc, pot); \
    return true;                                                                                                  \
  }
  FMMA_L2LP_CASE(4, 3) FMMA_L2LP_CASE(5, 3) FMMA_L2LP_CASE(6, 3) FMMA_L2LP_CASE(7, 3)
  FMMA_L2LP_CASE(4, 2) FMMA_L2LP_CASE(5, 2) FMMA_L2LP_CASE(6, 2) FMMA_L2LP_CASE(7, 2) FMMA_L2LP_CASE(8, 2)
#undef FMMA_L2LP_CASE
  return false;
}

void launch_lists_topdown(fmma_ctx* ctx, const Level& Lv, const Level* Pl, const int* pnbr, int d, int nfar,
                          const int* jslot, int* nbr, int* row_of_box, unsigned long long* pairs) {
  const int nnb = d == 1 ? 3 : (d == 2 ? 9 : 27);
  const int64_t nb = Lv.nbox;
  if (nb == 0) return;
  FMMA_CHECK_CUDA(cudaMemsetAsync(nbr, 0xff, sizeof(int) * (size_t)nb * nnb, ctx->stream));
  const int* rob = nullptr;
  if (Lv.nrow > 0) {
    FMMA_CHECK_CUDA(cudaMemsetAsync(row_of_box, 0xff, sizeof(int) * (size_t)nb, ctx->stream));
    FMMA_LAUNCH(ctx, k_rows_of_boxes, grid_for(Lv.nrow, 256), 256, 0, Lv.row_box, Lv.nrow, row_of_box);
    FMMA_CHECK_CUDA(cudaMemsetAsync(Lv.il, 0xff, sizeof(int) * (size_t)Lv.nrow * nfar, ctx->stream));
    FMMA_CHECK_CUDA(cudaMemsetAsync(Lv.slot_mask, 0, sizeof(unsigned) * (size_t)Lv.nrow * kSlotWords, ctx->stream));
    rob = row_of_box;
  }
  FMMA_LAUNCH(ctx, k_lists_topdown, grid_for(nb * nnb, 256, (int64_t)ctx->sm_count * 64), 256, 0, Lv.key, Lv.parent,
              nb, Lv.tb, Lv.te, Lv.v == 0, Lv.sb, Lv.se, pnbr, Pl ? Pl->cb : nullptr, Pl ? Pl->ce : nullptr, d, rob, nfar, jslot, nbr,
              Lv.il, Lv.slot_mask, pairs);
}

void launch_near_rows(fmma_ctx* ctx, const int* nbr, const int* row_box, int64_t nrow, int d, const int* sb,
                      const int* se, int* near) {
  const int nnb = d == 1 ? 3 : (d == 2 ? 9 : 27);
  if (nrow > 0)
    FMMA_LAUNCH(ctx, k_near_rows, grid_for(nrow * nnb, 256, (int64_t)ctx->sm_count * 64), 256, 0, nbr, row_box, nrow,
                nnb, sb, se, near);
}

}  // namespace fmma_b200
