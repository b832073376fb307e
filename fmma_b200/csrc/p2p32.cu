// p2p32.cu — mixed-precision near field: FP32 kernel evaluations on box-local
// coordinates, accumulated in FP32 with two-sum compensation (Knuth's TwoSum:
// an add also yields its exact rounding error, summed into a second FP32
// word), and the FP64 add of the far field.  Each lane sums at most
// kP2PBlock terms (16 in the target-lane kernel with 8 or 16 rhs per pass) in
// a plain FP32 partial, then folds the partial into its compensated (sum,
// error) pair with TwoSum; the pairs are added in FP64 across the warp.
//
// Same sum as src/fmm.cpp:121-141 (3^d near leaves of each target).  Points
// are stored relative to their own leaf centre as double-float pairs
// (hi + lo, both FP32); the target's offset to a neighbour box is formed once
// per (warp, box).  The difference x - y = (a_hi - y_hi) + (a_lo - y_lo) is
// then FP32 arithmetic whose first subtraction is exact for close points
// (Sterbenz), so each term keeps FP32 relative accuracy even when |x - y| is
// far below the leaf width.  With the compensated sums the accumulation adds
// an error of about one FP32 rounding of the running sum per lane, plus the
// roundings inside the short partials (at most kP2PBlock - 1 adds, the same
// order as the FP32 kernel evaluations of those terms), rather than one
// rounding of the running sum per term: the neighbour lists of dense leaves,
// thousands of sources, stay at the accuracy of the FP32 evaluations
// themselves.  Folding every kP2PBlock terms instead of every term keeps the
// compensation at ~1 extra operation per term and right-hand side.
#include <cuda_runtime.h>

#include "fmm_stages.cuh"
#include "fmma_internal.cuh"
#include "kernels.cuh"
#include "solver.cuh"

namespace fmma_b200 {

__device__ __forceinline__ void box_center(uint64_t key, int d, int bits, const Cube& c, double len, double* ctr) {
  int cc[kMaxDim] = {0, 0, 0};
  morton_decode(key, d, bits, cc);
  for (int q = 0; q < d; ++q) ctr[q] = c.origin[q] + len * ((double)cc[q] + 0.5);
}

// Double-float local coordinates of sorted points relative to their leaf
// centre: xl[q][j] = hi, xl[d + q][j] = lo with hi + lo = x - centre.
__global__ void k_local_coords(const uint64_t* __restrict__ key, const int* __restrict__ b0,
                               const int* __restrict__ b1, int64_t nbox, const double* __restrict__ x, int64_t n,
                               int d, const int* __restrict__ depth, const Cube* __restrict__ cubes,
                               float* __restrict__ xl) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.y + threadIdx.y; b < nbox; b += (int64_t)gridDim.x * blockDim.y) {
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int bits = depth[pid] - 1;
    const double len = c.Len / (double)(1 << bits);
    double ctr[kMaxDim];
    box_center(key[b] & kMortonMask, d, bits, c, len, ctr);
    for (int j = b0[b] + threadIdx.x; j < b1[b]; j += blockDim.x)
      for (int q = 0; q < d; ++q) {
        const double v = x[(int64_t)q * n + j] - ctr[q];
        const float hi = (float)v;
        xl[(int64_t)q * n + j] = hi;
        xl[(int64_t)(d + q) * n + j] = (float)(v - (double)hi);
      }
  }
}

// The same with one thread per leaf, for leaves holding a few points (the
// warp-per-leaf form above leaves most lanes idle there): consecutive
// threads take consecutive leaves, whose points are consecutive in memory.
__global__ void k_local_coords_tpl(const uint64_t* __restrict__ key, const int* __restrict__ b0,
                                   const int* __restrict__ b1, int64_t nbox, const double* __restrict__ x, int64_t n,
                                   int d, const int* __restrict__ depth, const Cube* __restrict__ cubes,
                                   float* __restrict__ xl) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbox; b += (int64_t)gridDim.x * blockDim.x) {
    const int j0 = b0[b], j1 = b1[b];
    if (j1 <= j0) continue;
    const int pid = key_pid(key[b]);
    const Cube& c = cubes[pid];
    const int bits = depth[pid] - 1;
    const double len = c.Len / (double)(1 << bits);
    double ctr[kMaxDim];
    box_center(key[b] & kMortonMask, d, bits, c, len, ctr);
    for (int j = j0; j < j1; ++j)
      for (int q = 0; q < d; ++q) {
        const double v = x[(int64_t)q * n + j] - ctr[q];
        const float hi = (float)v;
        xl[(int64_t)q * n + j] = hi;
        xl[(int64_t)(d + q) * n + j] = (float)(v - (double)hi);
      }
  }
}

// Sources staged per neighbour chunk, and the per-warp shared bytes: the
// FP64 sums (RB >= 8) and two staging buffers, each a chunk's weights and
// coordinates.
__host__ __device__ constexpr int p2p_chunk(int RB) { return RB >= 16 ? 32 : 64; }
__host__ __device__ constexpr size_t p2p_stage_bytes(int D, int RB) {
  return sizeof(float) * p2p_chunk(RB) * RB + sizeof(float) * 2 * D * p2p_chunk(RB);
}
__host__ __device__ constexpr size_t p2p_warp_bytes(int D, int RB) {
  return (RB >= 8 ? sizeof(double) * RB * 32 : 0) + 2 * p2p_stage_bytes(D, RB);
}

// s + c += t with TwoSum: s2 = fl(s + t) and e = (s + t) - s2 exactly (six
// FP32 operations, correct for any magnitudes); e goes into the compensation
// word c.  The _rn intrinsics keep the compiler from contracting or
// reassociating the sequence.
__device__ __forceinline__ void two_sum_acc(float& s, float& c, float t) {
  const float s2 = __fadd_rn(s, t);
  const float bp = __fsub_rn(s2, s);
  const float ap = __fsub_rn(s2, bp);
  c = __fadd_rn(c, __fadd_rn(__fsub_rn(s, ap), __fsub_rn(t, bp)));
  s = s2;
}

// terms per lane in a plain FP32 partial before it is folded by TwoSum
constexpr int kP2PBlock = 8;
// the target-lane kernel with 8 or 16 rhs per pass keeps its compensated pairs
// in shared memory (a fold is 2 * RB shared accesses): it folds every 16 terms
template <int RB>
constexpr int p2p_block() { return RB >= 8 ? 2 * kP2PBlock : kP2PBlock; }

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}

template <int KID, int D, int RB, typename T>
__global__ void __launch_bounds__(256, (D == 3 && RB == 16) ? 2 : 3) k_p2p_f32(
    const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ near, int nnear,
    const uint64_t* __restrict__ key, const int* __restrict__ tb, const int* __restrict__ te,
    const int* __restrict__ sb, const int* __restrict__ se, const float* __restrict__ txl, int64_t nt,
    const float* __restrict__ sxl, int64_t ns, const float* __restrict__ wst, int R, int Rp, float p0,
    const int* __restrict__ depth, const Cube* __restrict__ cubes, const double* __restrict__ pot,
    const int* __restrict__ perm_t, T* __restrict__ out) {
  // Per warp, in dynamic shared memory: the per-lane compensated FP32 sums
  // (sum, error) when the rhs block is wide (registers for up to 4 rhs;
  // keeps the kernel at 3 blocks per SM) and two staging buffers, each a
  // chunk's weights and coordinates (hi[D], lo[D]).
  constexpr int SC = p2p_chunk(RB);
  constexpr bool kSmemAcc = RB >= 8;
  extern __shared__ __align__(16) unsigned char p2p_smem[];
  const int lane = threadIdx.x & 31;
  unsigned char* wb = p2p_smem + (size_t)(threadIdx.x >> 5) * p2p_warp_bytes(D, RB);
  float2 (*scs)[32] = reinterpret_cast<float2 (*)[32]>(wb);
  // staging buffer b: weights sw[i][r] then coordinates sy[c][i]
  unsigned char* const stage0 = wb + (kSmemAcc ? sizeof(double) * RB * 32 : 0);
  auto sw_of = [&](int b) {
    return reinterpret_cast<float (*)[RB]>(stage0 + (size_t)b * p2p_stage_bytes(D, RB));
  };
  auto sy_of = [&](int b) {
    return reinterpret_cast<float (*)[SC]>(stage0 + (size_t)b * p2p_stage_bytes(D, RB) + sizeof(float) * SC * RB);
  };
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = wid; row < nrow; row += nw) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const double len = cubes[pid].Len / (double)(1 << (depth[pid] - 1));
    const int t0 = tb[b], t1 = te[b];
    for (int tc = t0; tc < t1; tc += 32) {
      // cnt targets on the low lanes, G source groups on the high ones
      const int cnt = min(32, t1 - tc);
      int tp2 = 1;
      while (tp2 < cnt) tp2 <<= 1;
      const int G = 32 / tp2;
      const int ti = lane & (tp2 - 1), g = lane / tp2;
      const bool tv = ti < cnt;
      double xd[D];
#pragma unroll
      for (int q = 0; q < D; ++q)
        xd[q] = tv ? (double)txl[(int64_t)q * nt + tc + ti] + (double)txl[(int64_t)(D + q) * nt + tc + ti] : 0.0;
      for (int r0 = 0; r0 < R; r0 += RB) {
        constexpr int RR = kSmemAcc ? 1 : RB;  // register pairs
        float cs[RR], ce[RR];                  // compensated sum and its error (RB <= 4)
#pragma unroll
        for (int r = 0; r < RR; ++r) cs[r] = ce[r] = 0.f;
        if (kSmemAcc) {
#pragma unroll
          for (int r = 0; r < RB; ++r) scs[r][lane] = make_float2(0.f, 0.f);
        }
        // The chunks of the 3^d neighbour leaves in order, chunk k + 1 copied
        // (cp.async) into the other buffer while chunk k is evaluated.
        // Cursor: neighbour slot q, chunk start c0, end of that leaf's sources je.
        auto advance = [&](int& q, int& c0, int& je) {
          c0 += SC;
          while (c0 >= je) {
            if (++q >= nnear) return false;
            const int sbx = near[row * nnear + q];  // warp-uniform
            if (sbx >= 0) {
              c0 = sb[sbx];
              je = se[sbx];
            }
          }
          return true;
        };
        auto stage = [&](int b, int c0, int je) {
          const int m = min(SC, je - c0);
          float (*syb)[SC] = sy_of(b);
          float (*swb)[RB] = sw_of(b);
#pragma unroll
          for (int c = 0; c < 2 * D; ++c)
            for (int i = lane; i < m; i += 32) cp_async4(&syb[c][i], sxl + (int64_t)c * ns + c0 + i);
          if constexpr (RB >= 4) {
            // rows of RB weights at 16-byte aligned offsets (Rp, r0: multiples of RB)
            constexpr int PV = RB / 4;
            for (int e = lane; e < m * PV; e += 32) {
              const int i = e / PV, pv = e - i * PV;
              cp_async16(&swb[i][4 * pv], wst + (int64_t)(c0 + i) * Rp + r0 + 4 * pv, true);
            }
          } else {
            for (int i = lane; i < m; i += 32) cp_async4(&swb[i][0], wst + (int64_t)(c0 + i) * Rp + r0);
          }
        };
        int cq = -1, cc0 = 0, cje = 0;
        bool have = advance(cq, cc0, cje);
        if (have) stage(0, cc0, cje);
        cp_async_commit();
        int buf = 0, prevq = -1;
        float ah[D], al[D];
        float part[RB];  // plain FP32 partial of at most p2p_block<RB>() terms
#pragma unroll
        for (int r = 0; r < RB; ++r) part[r] = 0.f;
        int nterm = 0;
        auto fold = [&]() {
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            if (kSmemAcc) {
              float2 sc = scs[r][lane];
              two_sum_acc(sc.x, sc.y, part[r]);
              scs[r][lane] = sc;
            } else {
              two_sum_acc(cs[kSmemAcc ? 0 : r], ce[kSmemAcc ? 0 : r], part[r]);
            }
            part[r] = 0.f;
          }
          nterm = 0;
        };
        while (have) {
          int nq = cq, nc0 = cc0, nje = cje;
          const bool hn = advance(nq, nc0, nje);
          if (hn) stage(buf ^ 1, nc0, nje);
          cp_async_commit();
          cp_async_wait<1>();  // this lane's copies of chunk k have landed
          __syncwarp();        // and every lane's
          if (cq != prevq) {
            prevq = cq;
            // the target relative to the centre of neighbour cq, whose offset
            // in leaf widths is the base-3 digits of cq minus one (near list
            // order, last dimension fastest)
            int qc = cq;
#pragma unroll
            for (int q = D - 1; q >= 0; --q) {
              const double av = xd[q] - len * (double)(qc % 3 - 1);
              qc /= 3;
              ah[q] = (float)av;
              al[q] = (float)(av - (double)ah[q]);
            }
          }
          const int m = min(SC, cje - cc0);
          const float (*sy)[SC] = sy_of(buf);
          const float (*sw)[RB] = sw_of(buf);
          if (tv) {
            for (int i = g; i < m; i += G) {
              float t[D];
#pragma unroll
              for (int q = 0; q < D; ++q) t[q] = (ah[q] - sy[q][i]) + (al[q] - sy[D + q][i]);
              const float f = keval_diff_f32<KID, D>(t, p0);
              if (RB == 1) {
                part[0] = fmaf(sw[i][0], f, part[0]);
              } else {
#pragma unroll
                for (int c4 = 0; c4 < RB / 4; ++c4) {
                  const float4 w4 = reinterpret_cast<const float4*>(&sw[i][0])[c4];
                  part[4 * c4 + 0] = fmaf(w4.x, f, part[4 * c4 + 0]);
                  part[4 * c4 + 1] = fmaf(w4.y, f, part[4 * c4 + 1]);
                  part[4 * c4 + 2] = fmaf(w4.z, f, part[4 * c4 + 2]);
                  part[4 * c4 + 3] = fmaf(w4.w, f, part[4 * c4 + 3]);
                }
              }
              if (++nterm == p2p_block<RB>()) fold();
            }
          }
          __syncwarp();  // buffer buf is restaged two chunks on
          buf ^= 1;
          cq = nq;
          cc0 = nc0;
          cje = nje;
          have = hn;
        }
        fold();
#pragma unroll
        for (int r = 0; r < RB; ++r) {
          double vr;
          if (kSmemAcc) {
            const float2 sc = scs[r][lane];
            vr = (double)sc.x + (double)sc.y;
          } else {
            vr = (double)cs[kSmemAcc ? 0 : r] + (double)ce[kSmemAcc ? 0 : r];
          }
          for (int o = tp2; o < 32; o <<= 1) vr += __shfl_xor_sync(0xffffffffu, vr, o);
          if (g == 0 && tv && r0 + r < R) {
            const int t = tc + ti;
            out[(int64_t)(r0 + r) * nt + perm_t[t]] = (T)(vr + (pot ? pot[(int64_t)(r0 + r) * nt + t] : 0.0));
          }
        }
      }
    }
  }
}

// Right-hand sides per pass: 1, 4, 8 or 16 (one pass for 9-16 right-hand
// sides, the kernel evaluated once per pair).  Every block width runs three
// 256-thread blocks per SM (80 registers; 8 and 16 keep their FP64 sums in
// shared memory), except 3-D with 16, whose sums and two staging buffers
// leave room for two (and so up to 128 registers for the 16 compensated
// FP32 sums).
// Sparse leaves (a few targets each, as in clustered sets at a uniform
// depth): lanes over the sources of the 3^d neighbour leaves taken as one
// list, targets looped.  Lane e finds its neighbour slot k from the prefix
// sums of the neighbours' source counts (a warp scan), re-expresses its
// source relative to the target leaf's centre once (FP64, split to FP32
// hi + lo, the same double-float form as the target), then evaluates FP32
// pairs against up to TB targets held in shared memory.  Per-lane compensated
// FP32 sums are added across the warp in FP64.
constexpr int kP2PSparseTB = 8;
// targets held per pass: 8 with one rhs, 4 with a block of 4 (the compensated
// sums of TB x RB pairs stay in registers)
__host__ __device__ constexpr int p2p_sparse_tb(int RB) { return RB == 1 ? kP2PSparseTB : kP2PSparseTB / 2; }

template <int KID, int D, int RB, typename T>
__global__ void __launch_bounds__(256, RB == 1 ? 4 : 2) k_p2p_f32_src(
    const int* __restrict__ row_box, int64_t nrow, const int* __restrict__ near, int nnear,
    const uint64_t* __restrict__ key, const int* __restrict__ tb, const int* __restrict__ te,
    const int* __restrict__ sb, const int* __restrict__ se, const float* __restrict__ txl, int64_t nt,
    const float* __restrict__ sxl, int64_t ns, const float* __restrict__ wst, int R, int Rp, float p0,
    const int* __restrict__ depth, const Cube* __restrict__ cubes, const double* __restrict__ pot,
    const int* __restrict__ perm_t, T* __restrict__ out, float2* __restrict__ cs_all) {
  constexpr int TB = p2p_sparse_tb(RB);
  __shared__ float s_x[256 / 32][TB][2 * D];  // per warp: target hi[D], lo[D]
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  // per lane: the compensated FP32 sums (sum, error) of the TB x RB (target,
  // rhs) pairs, in this warp's slice of a global scratch [warp][TB*RB][32]:
  // touched only by rows whose lanes take more than kP2PBlock sources, so
  // neither registers nor shared memory (the L1 share of the gathers) pay
  float2 (*s_cs)[32] = reinterpret_cast<float2 (*)[32]>(cs_all + wid * (TB * RB * 32));
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = wid; row < nrow; row += nw) {
    const int b = row_box[row];
    const int pid = key_pid(key[b]);
    const double len = cubes[pid].Len / (double)(1 << (depth[pid] - 1));
    // neighbour slot of this lane, its source range and the inclusive prefix of counts
    int box = -1, cnt = 0;
    if (lane < nnear) {
      box = near[row * nnear + lane];
      if (box >= 0) cnt = se[box] - sb[box];
    }
    int end = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, end, o);
      if (lane >= o) end += v;
    }
    const int total = __shfl_sync(0xffffffffu, end, 31);
    const int start = end - cnt;
    const int t0 = tb[b], t1 = te[b];
    for (int tc = t0; tc < t1; tc += TB) {
      const int ntg = min(TB, t1 - tc);
      __syncwarp();
      for (int e = lane; e < ntg * 2 * D; e += 32) {
        const int i = e / (2 * D), c = e - i * 2 * D;  // c < D: hi of dim c, else lo of dim c - D
        s_x[wib][i][c] = txl[(int64_t)c * nt + tc + i];
      }
      __syncwarp();
      // plain FP32 partials of at most kP2PBlock sources per lane (one source
      // per lane and pass of the loop below), folded by TwoSum into the
      // lane's compensated sums in shared memory when a row runs longer
      float part[TB][RB];
      auto fold = [&]() {
#pragma unroll
        for (int i = 0; i < TB; ++i)
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            float2 c = s_cs[i * RB + r][lane];
            two_sum_acc(c.x, c.y, part[i][r]);
            s_cs[i * RB + r][lane] = c;
            part[i][r] = 0.f;
          }
      };
      for (int r0 = 0; r0 < R; r0 += RB) {
#pragma unroll
        for (int i = 0; i < TB; ++i)
#pragma unroll
          for (int r = 0; r < RB; ++r) part[i][r] = 0.f;
        bool folded = false;  // warp-uniform
        int pass = 0;
        for (int e0 = 0; e0 < total; e0 += 32) {
          const int e = e0 + lane;
          // slot k: the number of neighbours whose range ends at or before e
          // (the ends are non-decreasing over the lanes: binary search)
          int k = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const int probe = k + step - 1;  // lanes >= nnear hold `total`, never <= e < total
            if (__shfl_sync(0xffffffffu, end, probe < 32 ? probe : 31) <= e && probe < nnear) k += step;
          }
          const int kq = min(k, 31);
          const int bk = __shfl_sync(0xffffffffu, box, kq);
          const int sk = __shfl_sync(0xffffffffu, start, kq);
          if (e < total) {
            const int j = sb[bk] + (e - sk);
            float yh[D], yl[D];
            int qc = k;
#pragma unroll
            for (int q = D - 1; q >= 0; --q) {
              // source relative to the target leaf's centre: own offset + len * (digit - 1)
              const double yv = ((double)sxl[(int64_t)q * ns + j] + (double)sxl[(int64_t)(D + q) * ns + j]) +
                                len * (double)(qc % 3 - 1);
              qc /= 3;
              yh[q] = (float)yv;
              yl[q] = (float)(yv - (double)yh[q]);
            }
            float w[RB];
            if (RB == 1) {
              w[0] = wst[(int64_t)j * Rp + r0];
            } else {
#pragma unroll
              for (int c4 = 0; c4 < RB / 4; ++c4) {
                const float4 w4 = reinterpret_cast<const float4*>(wst + (int64_t)j * Rp + r0)[c4];
                w[4 * c4] = w4.x; w[4 * c4 + 1] = w4.y; w[4 * c4 + 2] = w4.z; w[4 * c4 + 3] = w4.w;
              }
            }
#pragma unroll
            for (int i = 0; i < TB; ++i) {
              if (i < ntg) {
                float t[D];
#pragma unroll
                for (int q = 0; q < D; ++q) t[q] = (s_x[wib][i][q] - yh[q]) + (s_x[wib][i][D + q] - yl[q]);
                const float f = keval_diff_f32<KID, D>(t, p0);
#pragma unroll
                for (int r = 0; r < RB; ++r) part[i][r] = fmaf(w[r], f, part[i][r]);
              }
            }
          }
          if (++pass == kP2PBlock) {  // warp-uniform
            if (!folded) {
#pragma unroll
              for (int c = 0; c < TB * RB; ++c) s_cs[c][lane] = make_float2(0.f, 0.f);
              folded = true;
            }
            fold();
            pass = 0;
          }
        }
        if (folded) fold();
        // warp sums in FP64, then one lane per (target, rhs) writes
#pragma unroll
        for (int i = 0; i < TB; ++i) {
          if (i < ntg) {  // warp-uniform
#pragma unroll
            for (int r = 0; r < RB; ++r) {
              double v;
              if (folded) {
                const float2 c = s_cs[i * RB + r][lane];
                v = (double)c.x + (double)c.y;
              } else {
                v = (double)part[i][r];  // at most kP2PBlock terms: no fold needed
              }
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
              if (lane == i * RB + r && r0 + r < R) {
                const int t = tc + i;
                out[(int64_t)(r0 + r) * nt + perm_t[t]] = (T)(v + (pot ? pot[(int64_t)(r0 + r) * nt + t] : 0.0));
              }
            }
          }
        }
      }
    }
  }
}

static int p2p32_rhs_block(int R) { return R == 1 ? 1 : (R <= 4 ? 4 : (R <= 8 ? 8 : 16)); }

template <typename T>
struct P2P32Launch {
  template <int KID, int D>
  static void run(fmma_ctx* ctx, const Tree& tr, const float* txl, const float* sxl, const float* wst, int R, int Rp,
                  float p0, const double* pot, T* out) {
    const Level& Lf = tr.lev[0];
    const int nnear = D == 1 ? 3 : (D == 2 ? 9 : 27);
    unsigned g = grid_for(tr.nnear_rows * 32, 256, (int64_t)ctx->sm_count * 16);
    // sparse leaves and few right-hand sides: lanes over sources
    if (R <= 4 && tr.nt < (int64_t)kP2PSparseTB * tr.nnear_rows) {
      // compensated-sum scratch: per warp of the grid, TB x RB pairs per lane
      const size_t per_warp = (size_t)p2p_sparse_tb(R == 1 ? 1 : 4) * (R == 1 ? 1 : 4) * 32;
      float2* cs = ctx_buf_t<float2>(ctx, "p2p_cs", (size_t)g * (256 / 32) * per_warp);
      if (R == 1)
        FMMA_LAUNCH(ctx, (k_p2p_f32_src<KID, D, 1, T>), g, 256, 0, tr.near_row_box, tr.nnear_rows, tr.near, nnear,
                    Lf.key, Lf.tb, Lf.te, Lf.sb, Lf.se, txl, tr.nt, sxl, tr.ns, wst, R, Rp, p0, tr.d_depth, tr.d_cube,
                    pot, tr.perm_t, out, cs);
      else
        FMMA_LAUNCH(ctx, (k_p2p_f32_src<KID, D, 4, T>), g, 256, 0, tr.near_row_box, tr.nnear_rows, tr.near, nnear,
                    Lf.key, Lf.tb, Lf.te, Lf.sb, Lf.se, txl, tr.nt, sxl, tr.ns, wst, R, Rp, p0, tr.d_depth, tr.d_cube,
                    pot, tr.perm_t, out, cs);
      return;
    }
    switch (p2p32_rhs_block(R)) {
#define FMMA_P2P32_RB(RB_)                                                                                         \
  case RB_: {                                                                                                     \
    const size_t smem = p2p_warp_bytes(D, RB_) * 8;                                                              \
    static bool attr = false;                                                                                     \
    if (smem > 48 * 1024 && !attr && !ctx->capturing) {                                                           \
      FMMA_CHECK_CUDA(cudaFuncSetAttribute(k_p2p_f32<KID, D, RB_, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                           (int)smem));                                                           \
      attr = true;                                                                                                \
    }                                                                                                             \
    FMMA_LAUNCH(ctx, (k_p2p_f32<KID, D, RB_, T>), g, 256, smem, tr.near_row_box, tr.nnear_rows, tr.near, nnear,    \
                Lf.key, Lf.tb, Lf.te, Lf.sb, Lf.se, txl, tr.nt, sxl, tr.ns, wst, R, Rp, p0, tr.d_depth, tr.d_cube, \
                pot, tr.perm_t, out);                                                                             \
    break;                                                                                                        \
  }
      FMMA_P2P32_RB(1) FMMA_P2P32_RB(4) FMMA_P2P32_RB(8) FMMA_P2P32_RB(16)
#undef FMMA_P2P32_RB
      default: break;
    }
  }
};

// wst[j][r] = (float)ws[r][j] for r < R, zero for R <= r < Rp: the weights of
// one source are contiguous, read as float4.
__global__ void k_weights_f32_t(const double* __restrict__ ws, int R, int Rp, int64_t ns, float* __restrict__ wst) {
  const int64_t n = ns * Rp;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / Rp;
    const int r = (int)(e - j * Rp);
    wst[e] = r < R ? (float)ws[(int64_t)r * ns + j] : 0.f;
  }
}

// The sweep's weights in tree order in one pass: ws[r][j] = w[r][perm[j]] (1
// when w is null) in FP64 for the far field and, for the near field,
// wst[j][r] = (float)ws[r][j] for r < Rp (zero for r >= R), written as float4
// when Rp is a multiple of 4 (the same values k_weights_f32_t would form).
template <typename T>
__global__ void k_gather_weights_f32t(const T* __restrict__ w, const int* __restrict__ perm, int64_t ns, int R, int Rp,
                                      double* __restrict__ ws, float* __restrict__ wst) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pj = perm[j];
    auto val = [&](int r) {
      if (r >= R) return 0.0;
      const double v = w ? (double)w[(int64_t)r * ns + pj] : 1.0;
      ws[(int64_t)r * ns + j] = v;
      return v;
    };
    if (Rp % 4 == 0) {
      float4* dst = reinterpret_cast<float4*>(wst + j * Rp);
      for (int r = 0; r < Rp; r += 4) {
        float4 q;
        q.x = (float)val(r);
        q.y = (float)val(r + 1);
        q.z = (float)val(r + 2);
        q.w = (float)val(r + 3);
        dst[r / 4] = q;
      }
    } else {
      for (int r = 0; r < Rp; ++r) wst[j * Rp + r] = (float)val(r);
    }
  }
}

template <typename T>
void gather_weights_mixed(fmma_ctx* ctx, const T* w, const int* perm, int64_t ns, int R, double* ws) {
  const int RB = p2p32_rhs_block(R);
  const int Rp = (R + RB - 1) / RB * RB;
  float* wst = ctx_buf_t<float>(ctx, "wsf", (size_t)Rp * ns);
  if (ns > 0) FMMA_LAUNCH(ctx, k_gather_weights_f32t<T>, grid_for(ns, 256), 256, 0, w, perm, ns, R, Rp, ws, wst);
}

template void gather_weights_mixed<double>(fmma_ctx*, const double*, const int*, int64_t, int, double*);
template void gather_weights_mixed<float>(fmma_ctx*, const float*, const int*, int64_t, int, double*);

template <typename T>
void p2p_mixed(fmma_ctx* ctx, int d, const double* tx, const double* sx, const double* ws, int R, const double* pot,
               T* out, bool wst_ready) {
  Tree& tr = ctx->tree;
  const Level& Lf = tr.lev[0];
  float* txl = ctx_buf_t<float>(ctx, "txl", (size_t)(2 * d * tr.nt));
  float* sxl = ctx_buf_t<float>(ctx, "sxl", (size_t)(2 * d * tr.ns));
  const int RB = p2p32_rhs_block(R);
  const int Rp = (R + RB - 1) / RB * RB;
  float* wst = ctx_buf_t<float>(ctx, "wsf", (size_t)Rp * tr.ns);
  if (tr.nt + tr.ns < 16 * Lf.nbox) {  // a few points per leaf: one thread per leaf
    const unsigned g = grid_for(Lf.nbox, 256, (int64_t)ctx->sm_count * 16);
    FMMA_LAUNCH(ctx, k_local_coords_tpl, g, 256, 0, Lf.key, Lf.tb, Lf.te, Lf.nbox, tx, tr.nt, d, tr.d_depth, tr.d_cube,
                txl);
    FMMA_LAUNCH(ctx, k_local_coords_tpl, g, 256, 0, Lf.key, Lf.sb, Lf.se, Lf.nbox, sx, tr.ns, d, tr.d_depth, tr.d_cube,
                sxl);
  } else {
    dim3 blk(32, 8);
    FMMA_LAUNCH(ctx, k_local_coords, grid_for(Lf.nbox, 8, (int64_t)ctx->sm_count * 32), blk, 0, Lf.key, Lf.tb, Lf.te,
                Lf.nbox, tx, tr.nt, d, tr.d_depth, tr.d_cube, txl);
    FMMA_LAUNCH(ctx, k_local_coords, grid_for(Lf.nbox, 8, (int64_t)ctx->sm_count * 32), blk, 0, Lf.key, Lf.sb, Lf.se,
                Lf.nbox, sx, tr.ns, d, tr.d_depth, tr.d_cube, sxl);
  }
  if (!wst_ready)  // else gather_weights_mixed wrote them with the sweep's weights
    FMMA_LAUNCH(ctx, k_weights_f32_t, grid_for((int64_t)Rp * tr.ns, 256), 256, 0, ws, R, Rp, tr.ns, wst);
  dispatch_kernel<P2P32Launch<T>>(ctx->kernel_id, d, ctx, tr, txl, sxl, wst, R, Rp, (float)ctx->p0, pot, out);
}

template void p2p_mixed<double>(fmma_ctx*, int, const double*, const double*, const double*, int, const double*,
                                double*, bool);
template void p2p_mixed<float>(fmma_ctx*, int, const double*, const double*, const double*, int, const double*, float*,
                               bool);

}  // namespace fmma_b200
