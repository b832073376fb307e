// m2l_tc.cu — M2L on the 5th-generation tensor cores (tcgen05, sm_100a) with
// split-precision operands: D += A_hi B_hi + A_hi B_lo + A_lo B_hi, with
// A = gathered multipole coefficients and B = the slot's M2L operator, both
// split into TF32 (or BF16) high and low parts, accumulated in FP32 in TMEM.
// Tensor-core accumulation rounds toward zero, so the error grows with the
// number of MMA steps summed into one accumulator: every `group` slots the
// epilogue drains the (double-buffered) TMEM accumulator into FP32 registers
// (round to nearest) and the accumulator restarts.  Each row's running sum
// lives in the registers of three epilogue threads; Wl is written once per
// tile in FP64.  `group` (slots per drain), the pipeline depth cap and the
// units per stage are context options (fmma_set_m2l_options); A_hi, used by
// two products, is read from shared memory once and kept in the A collector
// for the second.  A pipeline stage holds up to four (slot, K chunk) units, so
// that one barrier wait and one MMA commit serve several units' MMAs: a
// commit costs the tensor pipe a few hundred cycles, as much as the six MMAs
// of a unit at small P.
//
// The contraction is the same as the FP64 path (src/fmm_core.cpp:383-455 in
// the reference: Wl[b] += K_{o(b,b')} Wm[b'] over the far list), organised as
// a GEMM per child-parity class: rows = target boxes x rhs (M = 128 per CTA
// tile), columns = output coefficients (N = P padded to 16), K = slots x P.
//
// CTA roles (544 threads, one CTA per SM, persistent over tiles):
//   warps 0..NPW-1   producers (NPW = 4, or 8 when N <= 96): cp.async gather
//               of A (hi/lo) into 64B-swizzled K-major smem, one bulk copy
//               per B part (pre-swizzled tables); cp.async delivery grows
//               with the warps that issue it, so small expansions, whose
//               epilogue needs fewer threads, take 8
//   warps NPW-15 epilogue: tcgen05.ld of the finished accumulator; warp w
//               reads TMEM lane quadrant w % 4 (32 rows) and one of the
//               (16 - NPW) / 4 column groups (at most 6 chunks of 16 columns
//               a thread), and keeps those sums in FP32 registers (a 16-warp
//               layout capped the kernel at 80 registers and measured 10 %
//               slower on the C3 leaf level)
//   warp 16     TMEM allocation and the single MMA-issuing thread
// Every mbarrier wait is bounded (TcParams::wait_cycles).  A wait that gives
// up raises the CTA's abort flag and sets the error flag that the host turns
// into FMMA_ERR_TIMEOUT; every role then stops at its next wait and drains
// before the CTA leaves: producers wait for their own gathers, complete the
// arrivals a warp still owes on stages that carry operator copies, and
// thread 0 waits for the last phase armed on each stage; the MMA issuer
// commits to a drain barrier and waits for it, so no copy or MMA is in
// flight when TMEM is freed.  (A separate barrier for the operator copies
// would make the drain simpler but costs the MMA issuer a second wait per
// stage: 15 % on the C3 leaf level.)
#include <cuda_bf16.h>

#include <cstdio>
#include <cstdlib>

#include "fmm_stages.cuh"
#include "fmma_internal.cuh"
#include "solver.cuh"

namespace fmma_b200 {

constexpr int kTcM = 128;
constexpr int kTcMaxStages = 8;
constexpr int kTcSmemMax = 232448;  // dynamic shared memory per block on sm_100
// Warp roles: NPW producer warps (4 or 8), 16 - NPW epilogue warps (column
// groups x 4 TMEM lane quadrants), warp 16 allocates TMEM and issues the MMAs.
constexpr int kTcMmaWarp = 16;
constexpr int kTcThreads = 32 * (kTcMmaWarp + 1);  // 544
template <int NPW>
struct TcRoles {
  static_assert(NPW == 4 || NPW == 8, "4 or 8 producer warps");
  static constexpr int PROD = 32 * NPW;         // producer threads
  static constexpr int RPW = 128 / NPW;         // tile rows per producer warp
  static constexpr int EPW = 16 - NPW;          // epilogue warps
  static constexpr int EG = EPW / 4;            // epilogue column groups
};
constexpr int kGroupSlotsDefault = 2;
constexpr int kDrainSteps = 84;  // MMA accumulation steps between drains (2 slots at P = 216)
constexpr long long kWaitCycles = 4000000000ll;  // ~2 s at 2 GHz
constexpr int kSlotPF = 8;                        // producers' source-box prefetch, in slots
constexpr int kTcMaxUnits = 4;                    // (slot, K chunk) units per pipeline stage, at most
constexpr int kTcStaticSmem = 3072;               // static shared memory of the kernels (upper bound)

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a phase parity.  False when `limit` SM clocks pass (the
// waiter then raises the CTA's abort flag) or when another thread of the CTA
// has raised it: every role stops at its next wait and drains.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit, volatile int* abort) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (*abort) return false;
    if (clock64() - t0 > limit) {
      *abort = 1;
      return false;
    }
  }
}
// The same wait during the drain that follows an abort: the copies and MMAs
// already issued finish on their own, so it waits for them with the default
// bound and ignores the abort flag.
__device__ __forceinline__ bool mbar_drain_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}
// Bounded wait for a device flag to become non-zero (the test hold).
__device__ __forceinline__ bool flag_wait(const int* flag, long long limit) {
  const long long t0 = clock64();
  while (*(const volatile int*)flag == 0)
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Arrive on `bar` once all cp.async operations this thread issued so far have
// completed; counts as one of the barrier's expected arrivals.
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
// COL: 0 = A read from shared memory and not kept, 1 = read and kept in the
// A collector buffer (fill), 2 = taken from the collector, which is then
// released (lastuse): two back-to-back MMAs on the same A read it once.
template <bool BF16, int COL = 0>
__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
#define FMMA_TC_MMA(KIND, COLQ)                                                                          \
  asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"                                               \
               "tcgen05.mma.cta_group::1.kind::" KIND COLQ " [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),       \
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)                                              \
               : "memory")
  if (BF16) {
    if (COL == 1) FMMA_TC_MMA("f16", ".collector::a::fill");
    else if (COL == 2) FMMA_TC_MMA("f16", ".collector::a::lastuse");
    else FMMA_TC_MMA("f16", "");
  } else {
    if (COL == 1) FMMA_TC_MMA("tf32", ".collector::a::fill");
    else if (COL == 2) FMMA_TC_MMA("tf32", ".collector::a::lastuse");
    else FMMA_TC_MMA("tf32", "");
  }
#undef FMMA_TC_MMA
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7, r8, r9, r10, r11, r12, r13, r14, r15;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7), "=r"(r8), "=r"(r9),
        "=r"(r10), "=r"(r11), "=r"(r12), "=r"(r13), "=r"(r14), "=r"(r15)
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7), "+r"(r8), "+r"(r9),
                 "+r"(r10), "+r"(r11), "+r"(r12), "+r"(r13), "+r"(r14), "+r"(r15)
               :
               : "memory");
  v[0] = __uint_as_float(r0); v[1] = __uint_as_float(r1); v[2] = __uint_as_float(r2); v[3] = __uint_as_float(r3);
  v[4] = __uint_as_float(r4); v[5] = __uint_as_float(r5); v[6] = __uint_as_float(r6); v[7] = __uint_as_float(r7);
  v[8] = __uint_as_float(r8); v[9] = __uint_as_float(r9); v[10] = __uint_as_float(r10); v[11] = __uint_as_float(r11);
  v[12] = __uint_as_float(r12); v[13] = __uint_as_float(r13); v[14] = __uint_as_float(r14); v[15] = __uint_as_float(r15);
}

// K-major operand in the canonical 64-byte swizzled layout: rows of 64 bytes,
// 8-row atoms of 512 bytes (SBO), start address advanced by 32 bytes per K
// step.
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;           // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;  // stride byte offset: next 8-row atom
  d |= (uint64_t)1 << 46;           // descriptor version for sm_100
  d |= (uint64_t)4 << 61;           // 64-byte swizzle
  return d;
}

// Instruction descriptor: D f32, A/B tf32 (2) or bf16 (1), both K-major.
__host__ __device__ constexpr uint32_t tc_idesc(bool bf16, int M, int N) {
  return (1u << 4) | ((bf16 ? 1u : 2u) << 7) | ((bf16 ? 1u : 2u) << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

template <bool BF16>
struct TcFmt {
  static constexpr int EL = BF16 ? 2 : 4;        // bytes per element
  static constexpr int ROW = 64;                 // bytes per K-chunk row
  static constexpr int CHUNK = ROW / EL;         // elements per chunk row
  static constexpr int KSTEP = BF16 ? 16 : 8;    // K per MMA (32 bytes)
  static constexpr int NSTEP = CHUNK / KSTEP;    // MMAs per chunk and product (2)
};

// byte offset of byte `ebyte` of row n inside a 64B-swizzled K-major block:
// the 16-byte unit index is XORed with bits 1-2 of the row
__host__ __device__ __forceinline__ int sw64_off(int n, int ebyte) {
  return n * 64 + ((((ebyte >> 4) ^ ((n >> 1) & 3)) << 4) | (ebyte & 15));
}

// ---------------------------------------------------------------------------
// split kernels
// ---------------------------------------------------------------------------
template <bool BF16>
__device__ __forceinline__ void split_store(double x, void* hi, void* lo) {
  if (BF16) {
    __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    *(__nv_bfloat16*)hi = h;
    *(__nv_bfloat16*)lo = l;
  } else {
    // TF32 = FP32 with the 13 low mantissa bits cleared; round half away
    // from zero on the magnitude bits, done explicitly on the bit pattern.
    const uint32_t h = (__float_as_uint((float)x) + 0x1000u) & 0xFFFFE000u;
    const float rem = (float)(x - (double)__uint_as_float(h));
    const uint32_t l = (__float_as_uint(rem) + 0x1000u) & 0xFFFFE000u;
    *(uint32_t*)hi = h;
    *(uint32_t*)lo = l;
  }
}

// Wm (FP64 [rows][Kpad64]) -> [rows][KCH][hi 64 B | lo 64 B] split elements,
// zero padded: the two halves of one K chunk of a row fill one 128-byte line.
// A thread converts 16 bytes' worth of consecutive elements and stores each
// half with one 16-byte store.
template <bool BF16>
__global__ void k_split_wm(const double* __restrict__ Wm, int64_t rows, int P, int Kpad64, int KpadTC,
                           char* __restrict__ out) {
  using F = TcFmt<BF16>;
  constexpr int VEC = 16 / F::EL;  // elements per 16-byte unit
  const int units = KpadTC / VEC;
  const int64_t total = rows * units;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = e / units;
    const int k0 = (int)(e - row * units) * VEC;
    uint4 hi, lo;
    char* h = reinterpret_cast<char*>(&hi);
    char* l = reinterpret_cast<char*>(&lo);
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int k = k0 + i;
      const double x = k < P ? Wm[row * Kpad64 + k] : 0.0;
      split_store<BF16>(x, h + i * F::EL, l + i * F::EL);
    }
    char* base = out + row * 2 * KpadTC * F::EL + (int64_t)(k0 / F::CHUNK) * 2 * F::ROW + (k0 % F::CHUNK) * F::EL;
    *reinterpret_cast<uint4*>(base) = hi;
    *reinterpret_cast<uint4*>(base + F::ROW) = lo;
  }
}

// FP64 table [noff][Npad64][Kpad64] -> [noff][KCH][2][Npad][64 B] swizzled blocks.
template <bool BF16>
__global__ void k_tc_table(const double* __restrict__ tab64, int P, int Npad64, int Kpad64, int noff, int KCH,
                           int Npad, char* __restrict__ out) {
  constexpr int EL = TcFmt<BF16>::EL, CH = TcFmt<BF16>::CHUNK;
  const int64_t total = (int64_t)noff * KCH * Npad * CH;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = e;
    const int c = (int)(t % CH); t /= CH;
    const int n = (int)(t % Npad); t /= Npad;
    const int kc = (int)(t % KCH); t /= KCH;
    const int64_t f = t;
    const int k = kc * CH + c;
    double x = (n < P && k < P) ? tab64[(f * Npad64 + n) * Kpad64 + k] : 0.0;
    const int64_t blk = (f * KCH + kc) * 2;
    const int64_t bbytes = (int64_t)Npad * TcFmt<BF16>::ROW;
    const int off = sw64_off(n, c * EL);
    split_store<BF16>(x, out + blk * bbytes + off, out + (blk + 1) * bbytes + off);
  }
}

// Non-empty slots of each tile, in slot order: one warp per tile ORs the
// slot bit sets of the tile's rows.
__global__ void k_tile_slots(const int4* __restrict__ tiles, int ntiles, const unsigned* __restrict__ slot_mask,
                             int nfar, int R, int* __restrict__ tile_nq, int* __restrict__ tile_q) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t tile = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntiles; tile += nw) {
    const int4 t = tiles[tile];
    const int b0 = t.y / R, b1 = (t.y + t.z - 1) / R;
    unsigned m[kSlotWords];
#pragma unroll
    for (int w = 0; w < kSlotWords; ++w) m[w] = 0u;
    for (int b = b0 + lane; b <= b1; b += 32)
#pragma unroll
      for (int w = 0; w < kSlotWords; ++w) m[w] |= slot_mask[(int64_t)b * kSlotWords + w];
    int base = 0;
#pragma unroll
    for (int w = 0; w < kSlotWords; ++w) {
      const unsigned word = __reduce_or_sync(0xffffffffu, m[w]);
      const int q = w * 32 + lane;
      const bool f = q < nfar && ((word >> lane) & 1u);
      const unsigned bal = __ballot_sync(0xffffffffu, f);
      if (f) tile_q[tile * nfar + base + __popc(bal & ((1u << lane) - 1u))] = q;
      base += __popc(bal);
    }
    if (lane == 0) tile_nq[tile] = base;
  }
}

// ---------------------------------------------------------------------------
// the tensor-core M2L kernel
// ---------------------------------------------------------------------------
struct TcParams {
  const int4* tiles;
  int ntiles;
  const int* tile_nq;
  const int* tile_q;
  const int* il;
  const int* row_box;
  const int* slot_off;
  const char* wms;   // split Wm rows
  const char* tab;   // split, swizzled operator blocks
  double* Wl;
  int P, Kpad64, KpadTC, KCH, Npad, nfar, R, tmem_cols, group, noff, stages;
  int units;       // (slot, K chunk) units per pipeline stage: one wait and one commit per stage
  int a_reuse;     // keep A_hi in the tensor core's A collector across its two products
  int nsplit;      // parts per tile (slot ranges); > 1 on levels with fewer tiles than SMs
  double* part;    // nsplit > 1: partial sums [tile * nsplit + part][kTcM][Npad]
  int* err;
  long long wait_cycles;  // bound of every pipeline wait (SM clocks)
  const int* hold;        // test hook: the MMA issuer first waits for this flag (null: no hold)
};

// Work item w = tile * nsplit + part covers slots [qa, qb) of the tile's list.
__device__ __forceinline__ void work_range(const TcParams& p, int w, int& tile, int& qa, int& qb) {
  tile = w / p.nsplit;
  const int part = w - tile * p.nsplit;
  const int nq = p.tile_nq[tile];
  qa = (int)((int64_t)part * nq / p.nsplit);
  qb = (int)((int64_t)(part + 1) * nq / p.nsplit);
}

// Pipeline stages of a work item of nq slots: each drain group of `group`
// slots is cut into stages of `units` consecutive (slot, K chunk) units; a
// stage never spans two groups.
__device__ __forceinline__ int item_stages(int nq, int group, int KCH, int units) {
  const int full = nq / group, rem = nq - full * group;
  return full * ((group * KCH + units - 1) / units) + (rem * KCH + units - 1) / units;
}

// Wl rows of the split tiles: the parts' partial sums added in part order.
__global__ void k_tc_split_sum(const int4* __restrict__ tiles, int ntiles, int nsplit, const double* __restrict__ part,
                               const int* __restrict__ row_box, int R, int Kpad64, int P, int Npad,
                               double* __restrict__ Wl) {
  const int64_t total = (int64_t)ntiles * kTcM * P;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t tr = e / P;
    const int col = (int)(e - tr * P);
    const int tile = (int)(tr / kTcM), row = (int)(tr - (int64_t)tile * kTcM);
    const int4 t = tiles[tile];
    if (row >= t.z) continue;
    double acc = 0.0;
    for (int k = 0; k < nsplit; ++k) acc += part[(((int64_t)tile * nsplit + k) * kTcM + row) * Npad + col];
    const int v = t.y + row;
    const int brow = v / R, r = v - brow * R;
    Wl[((int64_t)row_box[brow] * R + r) * Kpad64 + col] = acc;
  }
}

// Producers' drain (the PROD threads of the producer warps, after cp_async_wait<0>):
// after an abort a producer warp may have left before issuing its arrivals
// for stage uses that thread 0 already armed with operator copies; it makes
// those arrivals now (plain arrives, one per lane, as its cp.async arrivals
// would have been), so that each armed phase completes once its bytes land,
// and thread 0 waits for the phases it armed last on every stage.  Thread 0
// is at most S stage uses ahead of any warp (it waits on the empty barrier
// of the stage, which needs that warp's earlier arrivals), so the owed uses
// fall on distinct stages, each in its current phase.  `it` is the thread's
// count of stage uses issued.  Returns false when a wait gives up.
template <int PROD>
__device__ __forceinline__ bool producers_drain(uint64_t* full_bar, int S, int it, int* armed_sh) {
  const int tid = threadIdx.x;
  if (tid == 0) *armed_sh = it;
  asm volatile("bar.sync 1, %0;\n" ::"n"(PROD) : "memory");
  const int armed = *armed_sh;
  for (int u = it; u < armed; ++u) mbar_arrive(&full_bar[u % S]);
  asm volatile("bar.sync 1, %0;\n" ::"n"(PROD) : "memory");
  bool ok = true;
  if (tid == 0)
    for (int u = armed - S > 0 ? armed - S : 0; u < armed; ++u)
      ok = mbar_drain_wait(&full_bar[u % S], (uint32_t)(u / S) & 1u) && ok;
  return ok;
}

template <bool BF16, int CPT, int NPW>
__global__ void __launch_bounds__(kTcThreads, 1) k_m2l_tc(const TcParams p) {
  using F = TcFmt<BF16>;
  using RL = TcRoles<NPW>;
  extern __shared__ __align__(1024) char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kTcMaxStages], empty_bar[kTcMaxStages], accf_bar[2], acce_bar[2],
      drain_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;   // raised by the first wait that gives up
  __shared__ int armed_sh;   // stage uses armed by producer thread 0 (drain)
  __shared__ uint8_t s_slots[NPW][192];  // per producer warp: the current tile's slot ids

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  char* smem = (char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int S = p.stages, U = p.units;
  const int A_BYTES = kTcM * F::ROW;
  const int B_BYTES = p.Npad * F::ROW;
  const int UNIT = 2 * A_BYTES + 2 * B_BYTES;  // one (slot, K chunk) unit: A hi/lo, B hi/lo
  const int STAGE = U * UNIT;
  auto sA = [&](int st, int j, int part) { return smem + st * STAGE + j * UNIT + part * A_BYTES; };
  auto sB = [&](int st, int j, int part) { return smem + st * STAGE + j * UNIT + 2 * A_BYTES + part * B_BYTES; };

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], RL::PROD + 1);  // the producers' cp.async arrivals + the bulk expect_tx
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf_bar[b], 1);
      mbar_init(&acce_bar[b], RL::EPW * 32);
    }
    mbar_init(&drain_bar, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = tmem_base_sh;
  volatile int* abort = &abort_sh;
  const long long lim = p.wait_cycles;
  bool failed = false;

  if (warp < NPW) {
    // ---------------- producers ----------------
    // Warp w owns tile rows w * RPW ... (RPW = 32 or 16); lane l resolves the
    // source row of row w * RPW + l % RPW, and the copies are then spread so
    // that 8 lanes move one row's 128-byte line (hi and lo halves of the K
    // chunk): one copy instruction touches 4 lines, not 32.
    const int row_sub = lane >> 3, cpart = (lane >> 2) & 1, cunit = lane & 3;
    const int prow = warp * RL::RPW + (lane & (RL::RPW - 1));
    int it = 0;
    for (int w = blockIdx.x; w < p.ntiles * p.nsplit && !failed; w += gridDim.x) {
      int tile, qa, qb;
      work_range(p, w, tile, qa, qb);
      const int4 t = p.tiles[tile];
      const int cls = t.x, v0 = t.y, vcnt = t.z;
      const bool rv = prow < vcnt;
      int brow = 0, r = 0;
      if (rv) {
        int v = v0 + prow;
        brow = v / p.R;
        r = v - brow * p.R;
      }
      const int* tq = p.tile_q + (int64_t)tile * p.nfar;
      const int* ilrow = p.il + (int64_t)brow * p.nfar;
      // The tile's slot list is staged in this warp's shared-memory copy, and
      // each thread's source boxes for the next kSlotPF slots are loaded into
      // a register queue, so no chain of dependent global loads stands
      // between two slots (a slot is a single stage at small P).
      uint8_t* wq = s_slots[warp];
      for (int i = lane; i < qb - qa; i += 32) wq[i] = (uint8_t)tq[qa + i];
      __syncwarp();
      const int nqs = qb - qa;
      int sq[kSlotPF];
#pragma unroll
      for (int k = 0; k < kSlotPF; ++k) sq[k] = (k < nqs && rv) ? ilrow[wq[k]] : -1;
      // units (slot ql, chunk kc) in order; a stage takes up to U of a group's
      int ql = -1, kc = p.KCH - 1, f = 0;
      int64_t own = -1;  // source line base of this thread's own row (byte offset, -1 = empty)
      const int ngroups = (nqs + p.group - 1) / p.group;
      for (int g = 0; g < ngroups && !failed; ++g) {
        const int nu = (min(nqs, (g + 1) * p.group) - g * p.group) * p.KCH;
        for (int u0 = 0; u0 < nu; u0 += U) {
          const int un = min(U, nu - u0);
          const int st = it % S;
          const uint32_t n = (uint32_t)(it / S);
          const bool ok = __all_sync(0xffffffffu, mbar_wait(&empty_bar[st], (n & 1u) ^ 1u, lim, abort));
          if (!ok) { failed = true; break; }
          if (tid == 0) mbar_arrive_expect_tx(&full_bar[st], 2u * (uint32_t)B_BYTES * (uint32_t)un);
#pragma unroll
          for (int j = 0; j < kTcMaxUnits; ++j) {
            if (j >= un) break;
            if (++kc == p.KCH) {  // next slot
              kc = 0;
              ++ql;
              f = p.slot_off[cls * 189 + wq[ql]] + t.w * p.noff;
              const int s = sq[0];
#pragma unroll
              for (int k = 0; k + 1 < kSlotPF; ++k) sq[k] = sq[k + 1];
              sq[kSlotPF - 1] = (ql + kSlotPF < nqs && rv) ? ilrow[wq[ql + kSlotPF]] : -1;
              own = s >= 0 ? ((int64_t)s * p.R + r) * 2 * p.KpadTC * F::EL : -1;
            }
            if (tid == 0) {
              const char* tb = p.tab + (((int64_t)f * p.KCH + kc) * 2) * (int64_t)B_BYTES;
              bulk_g2s(sB(st, j, 0), tb, (uint32_t)B_BYTES, &full_bar[st]);
              bulk_g2s(sB(st, j, 1), tb + B_BYTES, (uint32_t)B_BYTES, &full_bar[st]);
            }
            const int64_t koff = (int64_t)kc * 2 * F::ROW + cpart * F::ROW + cunit * 16;
            char* dst = sA(st, j, cpart);
#pragma unroll
            for (int i = 0; i < RL::RPW / 4; ++i) {
              const int rl = 4 * i + row_sub;  // row within the warp's RPW
              const long long base = __shfl_sync(0xffffffffu, (long long)own, rl);
              const int row = warp * RL::RPW + rl;
              cp_async16(dst + sw64_off(row, cunit * 16), p.wms + (base >= 0 ? base + koff : 0), base >= 0);
            }
          }
          cp_async_arrive_noinc(&full_bar[st]);
          ++it;
        }
      }
    }
    // drain: every copy issued has landed before the CTA leaves
    cp_async_wait<0>();
    if (!producers_drain<RL::PROD>(full_bar, S, it, &armed_sh)) failed = true;
  } else if (warp < NPW + RL::EPW) {
    // ---------------- epilogue ----------------
    const int quad = warp & 3;              // TMEM lane quadrant = row block
    const int cgrp = (warp - NPW) >> 2;     // column group
    const int row = quad * 32 + lane;
    const int nch = p.Npad / 16;            // 16-column chunks
    const int c_lo = (nch * cgrp) / RL::EG, c_hi = (nch * (cgrp + 1)) / RL::EG;
    int gg = 0;
    for (int w = blockIdx.x; w < p.ntiles * p.nsplit && !failed; w += gridDim.x) {
      int tile, qa, qb;
      work_range(p, w, tile, qa, qb);
      const int4 t = p.tiles[tile];
      const bool rv = row < t.z;
      double* dst = nullptr;
      if (rv) {
        if (p.nsplit > 1) {
          dst = p.part + ((int64_t)w * kTcM + row) * p.Npad;
        } else {
          int v = t.y + row;
          int brow = v / p.R, r = v - brow * p.R;
          dst = p.Wl + ((int64_t)p.row_box[brow] * p.R + r) * p.Kpad64;
        }
      }
      float acc[CPT][16];
#pragma unroll
      for (int c = 0; c < CPT; ++c)
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c][j] = 0.f;
      const int ngroups = (qb - qa + p.group - 1) / p.group;
      for (int g = 0; g < ngroups; ++g) {
        const int b = gg & 1;
        const uint32_t m = (uint32_t)(gg >> 1);
        if (!mbar_wait(&accf_bar[b], m & 1u, lim, abort)) { failed = true; break; }
        tc_fence_after();
        const uint32_t tb = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * p.Npad);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (c_lo + c < c_hi) {
            float v[16];
            tmem_ld16(tb + (uint32_t)((c_lo + c) * 16), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[c][j] += v[j];
          }
        }
        tc_fence_before();
        mbar_arrive(&acce_bar[b]);
        ++gg;
      }
      if (rv) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (c_lo + c < c_hi) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int col = (c_lo + c) * 16 + j;
              if (col < p.P) dst[col] = (double)acc[c][j];
            }
          }
        }
      }
    }
  } else if (lane == 0) {
    // ---------------- MMA issuer ----------------
    const uint32_t idesc = tc_idesc(BF16, kTcM, p.Npad);
    int it = 0, gg = 0;
    if (p.hold && !flag_wait(p.hold, lim)) {
      *abort = 1;
      failed = true;
    }
    for (int w = blockIdx.x; w < p.ntiles * p.nsplit && !failed; w += gridDim.x) {
      int tile, qa, qb;
      work_range(p, w, tile, qa, qb);
      const int ngroups = (qb - qa + p.group - 1) / p.group;
      for (int g = 0; g < ngroups && !failed; ++g) {
        const int b = gg & 1;
        const uint32_t m = (uint32_t)(gg >> 1);
        if (!mbar_wait(&acce_bar[b], (m & 1u) ^ 1u, lim, abort)) { failed = true; break; }
        tc_fence_after();
        const uint32_t dt = tmem_base + (uint32_t)(b * p.Npad);
        const int nu = (min(qb - qa, (g + 1) * p.group) - g * p.group) * p.KCH;
        for (int u0 = 0; u0 < nu && !failed; u0 += U) {
          const int un = min(U, nu - u0);
          const int st = it % S;
          const uint32_t n = (uint32_t)(it / S);
          if (!mbar_wait(&full_bar[st], n & 1u, lim, abort)) {
            failed = true;
            break;
          }
          // no proxy fence between the cp.async barrier and the MMAs: the
          // cp.async arrive-on completes after the data is in shared memory
          // (as in CUTLASS's cp.async tcgen05 mainloop); a fence per stage on
          // this thread would sit on the MMA issue path
          tc_fence_after();
#pragma unroll
          for (int j = 0; j < kTcMaxUnits; ++j) {
            if (j >= un) break;
            const uint32_t ah = smem_u32(sA(st, j, 0)), al = smem_u32(sA(st, j, 1));
            const uint32_t bh = smem_u32(sB(st, j, 0)), bl = smem_u32(sB(st, j, 1));
#pragma unroll
            for (int ks = 0; ks < F::NSTEP; ++ks) {
              const uint32_t kb = (uint32_t)(ks * 32);
              const uint32_t first = (u0 + j == 0 && ks == 0) ? 0u : 1u;
              tc_mma<BF16>(dt, sdesc_sw64(al + kb), sdesc_sw64(bh + kb), idesc, first);
              if (p.a_reuse) {
                tc_mma<BF16, 1>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bl + kb), idesc, 1u);
                tc_mma<BF16, 2>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bh + kb), idesc, 1u);
              } else {
                tc_mma<BF16>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bl + kb), idesc, 1u);
                tc_mma<BF16>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bh + kb), idesc, 1u);
              }
            }
          }
          tc_commit(&empty_bar[st]);
          ++it;
        }
        tc_commit(&accf_bar[b]);
        ++gg;
      }
    }
    // drain: every MMA issued has completed (commit tracks all prior
    // tcgen05 operations of this thread) before TMEM is released
    tc_commit(&drain_bar);
    if (!mbar_drain_wait(&drain_bar, 0u)) failed = true;
  }

  if (failed) atomicOr(p.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == kTcMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// the 2-SM variant: a cluster of two CTAs on an SM pair, M = 256
// ---------------------------------------------------------------------------
// The same contraction with tcgen05 `cta_group::2`: one MMA instruction covers
// a 256-row tile, rows 0-127 from CTA 0's shared memory and 128-255 from CTA
// 1's, and the operator's N columns split between them (N/2 each), so per SM
// every MMA reads half the operator bytes and each stage loads half the
// operator: fewer shared-memory operand bytes and fewer L2 fills per flop than
// two 128-row CTAs.  Each CTA's TMEM holds the accumulator of its own 128
// rows over all N columns, which its own epilogue drains.
//
// Roles per CTA as in k_m2l_tc.  CTA 0 issues the MMAs.  Completion of CTA
// 1's stages reaches CTA 0's full barrier through a relay: CTA 1's producers
// arrive on its local barriers (cp.async arrive-on, bulk expect_tx), and one
// thread of CTA 1 (lane 0 of its otherwise idle MMA warp) waits for each
// stage in order and arrives on CTA 0's barrier.  The MMA
// commits reach both CTAs' empty and accumulator barriers by multicast; each
// epilogue warp of both CTAs arrives once on CTA 0's accumulator-empty
// barrier.  TMEM is allocated and freed by the same warp in both CTAs.
// Every wait is bounded as in k_m2l_tc; both CTAs meet at a cluster barrier
// before TMEM is freed, so no remote arrive or MMA targets a CTA that left.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
// shared::cluster address of the same variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
// Arrive on an mbarrier of another CTA of the cluster (release at CTA scope,
// the form of the 2-SM arrive in CUTLASS; a release at cluster scope made the
// relay the kernel's bottleneck: 25.7 against 17.6 ms on a 1.5M-point level).
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tc2_commit_both(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}
__device__ __forceinline__ void tc2_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
template <bool BF16, int COL = 0>
__device__ __forceinline__ void tc2_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
#define FMMA_TC2_MMA(KIND, COLQ)                                                                         \
  asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"                                               \
               "tcgen05.mma.cta_group::2.kind::" KIND COLQ " [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),       \
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)                                              \
               : "memory")
  if (BF16) {
    if (COL == 1) FMMA_TC2_MMA("f16", ".collector::a::fill");
    else if (COL == 2) FMMA_TC2_MMA("f16", ".collector::a::lastuse");
    else FMMA_TC2_MMA("f16", "");
  } else {
    if (COL == 1) FMMA_TC2_MMA("tf32", ".collector::a::fill");
    else if (COL == 2) FMMA_TC2_MMA("tf32", ".collector::a::lastuse");
    else FMMA_TC2_MMA("tf32", "");
  }
#undef FMMA_TC2_MMA
}

constexpr int kTc2M = 2 * kTcM;  // rows of a 2-SM tile

template <bool BF16, int CPT, int NPW>
__global__ void __launch_bounds__(kTcThreads, 1) k_m2l_tc2(const TcParams p) {
  using F = TcFmt<BF16>;
  using RL = TcRoles<NPW>;
  extern __shared__ __align__(1024) char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kTcMaxStages], empty_bar[kTcMaxStages], accf_bar[2], acce_bar[2],
      drain_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  __shared__ int armed_sh;
  __shared__ uint8_t s_slots[NPW][192];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank();
  const int cid = (int)(blockIdx.x >> 1), ncl = (int)(gridDim.x >> 1);
  char* smem = (char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int S = p.stages, U = p.units;
  const int NH = p.Npad / 2;  // operator rows held by this CTA
  const int A_BYTES = kTcM * F::ROW;
  const int B_BYTES = NH * F::ROW;
  const int BLK = p.Npad * F::ROW;  // one (hi or lo) operator block in global memory
  const int UNIT = 2 * A_BYTES + 2 * B_BYTES;
  const int STAGE = U * UNIT;
  auto sA = [&](int st, int j, int part) { return smem + st * STAGE + j * UNIT + part * A_BYTES; };
  auto sB = [&](int st, int j, int part) { return smem + st * STAGE + j * UNIT + 2 * A_BYTES + part * B_BYTES; };

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      // the producer arrivals + this CTA's operator expect_tx, and on CTA 0
      // the relay of CTA 1's stage
      mbar_init(&full_bar[s], rank == 0 ? RL::PROD + 2 : RL::PROD + 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf_bar[b], 1);
      mbar_init(&acce_bar[b], 2 * RL::EPW);  // one arrival per epilogue warp of both CTAs (CTA 0's copy)
    }
    mbar_init(&drain_bar, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs' barriers initialised and TMEM allocated
  tc_fence_after();
  const uint32_t tmem_base = tmem_base_sh;
  volatile int* abort = &abort_sh;
  const long long lim = p.wait_cycles;
  bool failed = false;
  const int nwork = p.ntiles;

  if (warp < NPW) {
    // ---------------- producers (both CTAs): rows rank*128 + warp*RPW + lane%RPW ----------------
    const int row_sub = lane >> 3, cpart = (lane >> 2) & 1, cunit = lane & 3;
    int it = 0;
    const int myrow = (int)rank * kTcM + warp * RL::RPW + (lane & (RL::RPW - 1));
    for (int w = cid; w < nwork && !failed; w += ncl) {
      const int tile = w, qa = 0, qb = p.tile_nq[w];
      const int4 t = p.tiles[tile];
      const int cls = t.x, v0 = t.y, vcnt = t.z;
      const bool rv = myrow < vcnt;
      int brow = 0, r = 0;
      if (rv) {
        const int v = v0 + myrow;
        brow = v / p.R;
        r = v - brow * p.R;
      }
      const int* tq = p.tile_q + (int64_t)tile * p.nfar;
      const int* ilrow = p.il + (int64_t)brow * p.nfar;
      uint8_t* wq = s_slots[warp];
      for (int i = lane; i < qb - qa; i += 32) wq[i] = (uint8_t)tq[qa + i];
      __syncwarp();
      const int nqs = qb - qa;
      int sq[kSlotPF];
#pragma unroll
      for (int k = 0; k < kSlotPF; ++k) sq[k] = (k < nqs && rv) ? ilrow[wq[k]] : -1;
      int ql = -1, kc = p.KCH - 1, f = 0;
      int64_t own = -1;
      const int ngroups = (nqs + p.group - 1) / p.group;
      for (int g = 0; g < ngroups && !failed; ++g) {
        const int nu = (min(nqs, (g + 1) * p.group) - g * p.group) * p.KCH;
        for (int u0 = 0; u0 < nu; u0 += U) {
          const int un = min(U, nu - u0);
          const int st = it % S;
          const uint32_t n = (uint32_t)(it / S);
          const bool ok = __all_sync(0xffffffffu, mbar_wait(&empty_bar[st], (n & 1u) ^ 1u, lim, abort));
          if (!ok) { failed = true; break; }
          if (tid == 0) mbar_arrive_expect_tx(&full_bar[st], 2u * (uint32_t)B_BYTES * (uint32_t)un);
#pragma unroll
          for (int j = 0; j < kTcMaxUnits; ++j) {
            if (j >= un) break;
            if (++kc == p.KCH) {  // next slot
              kc = 0;
              ++ql;
              f = p.slot_off[cls * 189 + wq[ql]] + t.w * p.noff;
              const int s = sq[0];
#pragma unroll
              for (int k = 0; k + 1 < kSlotPF; ++k) sq[k] = sq[k + 1];
              sq[kSlotPF - 1] = (ql + kSlotPF < nqs && rv) ? ilrow[wq[ql + kSlotPF]] : -1;
              own = s >= 0 ? ((int64_t)s * p.R + r) * 2 * p.KpadTC * F::EL : -1;
            }
            if (tid == 0) {  // this CTA's half of the operator block (pre-swizzled rows rank*NH ...)
              const char* tb = p.tab + (((int64_t)f * p.KCH + kc) * 2) * (int64_t)BLK + (int64_t)rank * B_BYTES;
              bulk_g2s(sB(st, j, 0), tb, (uint32_t)B_BYTES, &full_bar[st]);
              bulk_g2s(sB(st, j, 1), tb + BLK, (uint32_t)B_BYTES, &full_bar[st]);
            }
            const int64_t koff = (int64_t)kc * 2 * F::ROW + cpart * F::ROW + cunit * 16;
            char* dst = sA(st, j, cpart);
#pragma unroll
            for (int i = 0; i < RL::RPW / 4; ++i) {
              const int rl = 4 * i + row_sub;
              const long long base = __shfl_sync(0xffffffffu, (long long)own, rl);
              const int row = warp * RL::RPW + rl;
              cp_async16(dst + sw64_off(row, cunit * 16), p.wms + (base >= 0 ? base + koff : 0), base >= 0);
            }
          }
          cp_async_arrive_noinc(&full_bar[st]);
          ++it;
        }
      }
    }
    cp_async_wait<0>();
    if (!producers_drain<RL::PROD>(full_bar, S, it, &armed_sh)) failed = true;
  } else if (warp < NPW + RL::EPW) {
    // ---------------- epilogue (both CTAs): this CTA's 128 rows ----------------
    const int quad = warp & 3;
    const int cgrp = (warp - NPW) >> 2;
    const int lrow = quad * 32 + lane;
    const int row = (int)rank * kTcM + lrow;
    const int nch = p.Npad / 16;
    const int c_lo = (nch * cgrp) / RL::EG, c_hi = (nch * (cgrp + 1)) / RL::EG;
    const uint32_t acce0[2] = {map_to_rank(&acce_bar[0], 0), map_to_rank(&acce_bar[1], 0)};
    int gg = 0;
    for (int w = cid; w < nwork && !failed; w += ncl) {
      const int4 t = p.tiles[w];
      const int qb = p.tile_nq[w];
      const bool rv = row < t.z;
      double* dst = nullptr;
      if (rv) {
        const int v = t.y + row;
        const int brow = v / p.R, r = v - brow * p.R;
        dst = p.Wl + ((int64_t)p.row_box[brow] * p.R + r) * p.Kpad64;
      }
      float acc[CPT][16];
#pragma unroll
      for (int c = 0; c < CPT; ++c)
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c][j] = 0.f;
      const int ngroups = (qb + p.group - 1) / p.group;
      for (int g = 0; g < ngroups; ++g) {
        const int b = gg & 1;
        const uint32_t m = (uint32_t)(gg >> 1);
        if (!mbar_wait(&accf_bar[b], m & 1u, lim, abort)) { failed = true; break; }
        tc_fence_after();
        const uint32_t tb = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * p.Npad);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (c_lo + c < c_hi) {
            float v[16];
            tmem_ld16(tb + (uint32_t)((c_lo + c) * 16), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[c][j] += v[j];
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(acce0[b]);
        ++gg;
      }
      if (rv) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (c_lo + c < c_hi) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int col = (c_lo + c) * 16 + j;
              if (col < p.P) dst[col] = (double)acc[c][j];
            }
          }
        }
      }
    }
  } else if (lane == 0 && rank == 0) {
    // ---------------- MMA issuer (CTA 0) ----------------
    const uint32_t idesc = tc_idesc(BF16, kTc2M, p.Npad);
    int it = 0, gg = 0;
    if (p.hold && !flag_wait(p.hold, lim)) {
      *abort = 1;
      failed = true;
    }
    for (int w = cid; w < nwork && !failed; w += ncl) {
      const int qb = p.tile_nq[w];
      const int ngroups = (qb + p.group - 1) / p.group;
      for (int g = 0; g < ngroups && !failed; ++g) {
        const int b = gg & 1;
        const uint32_t m = (uint32_t)(gg >> 1);
        if (!mbar_wait(&acce_bar[b], (m & 1u) ^ 1u, lim, abort)) { failed = true; break; }
        tc_fence_after();
        const uint32_t dt = tmem_base + (uint32_t)(b * p.Npad);
        const int nu = (min(qb, (g + 1) * p.group) - g * p.group) * p.KCH;
        for (int u0 = 0; u0 < nu && !failed; u0 += U) {
          const int un = min(U, nu - u0);
          const int st = it % S;
          const uint32_t n = (uint32_t)(it / S);
          if (!mbar_wait(&full_bar[st], n & 1u, lim, abort)) {
            failed = true;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int j = 0; j < kTcMaxUnits; ++j) {
            if (j >= un) break;
            const uint32_t ah = smem_u32(sA(st, j, 0)), al = smem_u32(sA(st, j, 1));
            const uint32_t bh = smem_u32(sB(st, j, 0)), bl = smem_u32(sB(st, j, 1));
#pragma unroll
            for (int ks = 0; ks < F::NSTEP; ++ks) {
              const uint32_t kb = (uint32_t)(ks * 32);
              const uint32_t first = (u0 + j == 0 && ks == 0) ? 0u : 1u;
              tc2_mma<BF16>(dt, sdesc_sw64(al + kb), sdesc_sw64(bh + kb), idesc, first);
              tc2_mma<BF16, 1>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bl + kb), idesc, 1u);
              tc2_mma<BF16, 2>(dt, sdesc_sw64(ah + kb), sdesc_sw64(bh + kb), idesc, 1u);
            }
          }
          tc2_commit_both(&empty_bar[st]);
          ++it;
        }
        tc2_commit_both(&accf_bar[b]);
        ++gg;
      }
    }
    tc2_commit(&drain_bar);
    if (!mbar_drain_wait(&drain_bar, 0u)) failed = true;
  } else if (lane == 0) {
    // ---------------- relay (CTA 1): its stages, in order, to CTA 0 ----------------
    int it = 0;
    for (int w = cid; w < nwork && !failed; w += ncl) {
      const int nst = item_stages(p.tile_nq[w], p.group, p.KCH, U);
      for (int k = 0; k < nst; ++k) {
        const int st = it % S;
        const uint32_t n = (uint32_t)(it / S);
        if (!mbar_wait(&full_bar[st], n & 1u, lim, abort)) {
          failed = true;
          break;
        }
        mbar_arrive_cluster(map_to_rank(&full_bar[st], 0));
        ++it;
      }
    }
  }

  if (failed) atomicOr(p.err, 1);
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // CTA 0's MMAs are drained and no remote arrive is pending
  if (warp == kTcMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host side: one level
// ---------------------------------------------------------------------------
int tc_npad(int P) { return (P + 15) / 16 * 16; }

template <bool BF16, int CPT, int NPW>
static void launch_tc(fmma_ctx* ctx, unsigned grid, size_t smem, const TcParams& prm) {
  static size_t attr = 0;
  if (attr < smem && !ctx->capturing) {
    FMMA_CHECK_CUDA(
        cudaFuncSetAttribute(k_m2l_tc<BF16, CPT, NPW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = smem;
  }
  FMMA_LAUNCH(ctx, (k_m2l_tc<BF16, CPT, NPW>), grid, kTcThreads, smem, prm);
}

// 2-SM kernel: cluster launch of 2 CTAs per SM pair; the number of clusters
// that fit at once is queried once per instantiation and shared-memory size.
template <bool BF16, int CPT, int NPW>
static int tc2_max_clusters(fmma_ctx* ctx, size_t smem) {
  static size_t attr = 0;
  static int cached = 0;
  if (ctx->capturing) return attr >= smem ? cached : -1;  // no attribute changes inside a capture
  if (attr < smem) {
    FMMA_CHECK_CUDA(
        cudaFuncSetAttribute(k_m2l_tc2<BF16, CPT, NPW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = smem;
    cached = 0;
  }
  if (cached == 0) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(2 * (ctx->sm_count / 2)));
    cfg.blockDim = dim3(kTcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_m2l_tc2<BF16, CPT, NPW>, &cfg) != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    cached = n > 0 ? n : -1;
  }
  return cached;
}

template <bool BF16, int CPT, int NPW>
static void launch_tc2(fmma_ctx* ctx, int nclusters, size_t smem, const TcParams& prm) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(2 * nclusters));
  cfg.blockDim = dim3(kTcThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  FMMA_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_m2l_tc2<BF16, CPT, NPW>, prm));
  after_launch(ctx);
}

template <bool BF16>
static void m2l_level_tc_t(fmma_ctx* ctx, int pair_pref, int units_pref, const Level& Lv, int v, int nfar,
                           const int* slot_off, int P,
                           int Kpad64,
                           int R, const double* Wm64, double* Wl64, const double* tab64, int Npad64,
                           const std::string& tabkey, int noff, int ntab) {
  using F = TcFmt<BF16>;
  const int KpadTC = (P + F::CHUNK - 1) / F::CHUNK * F::CHUNK;
  const int KCH = KpadTC / F::CHUNK;
  const int Npad = tc_npad(P);
  FMMA_REQUIRE(Npad <= 256, "tensor-core M2L supports at most 256 coefficients per box");

  // split operator blocks (cached with the FP64 table)
  bool fresh = false;
  const size_t tab_bytes = (size_t)ntab * noff * KCH * 2 * Npad * F::ROW;
  char* tab = (char*)cached_op(ctx, tabkey + (BF16 ? "_bf16" : "_tf32"), tab_bytes, &fresh);
  if (fresh) {  // the ntab tables are contiguous: one conversion over ntab * noff operators
    int64_t total = (int64_t)ntab * noff * KCH * Npad * F::CHUNK;
    FMMA_LAUNCH(ctx, k_tc_table<BF16>, grid_for(total, 256, (int64_t)ctx->sm_count * 32), 256, 0, tab64, P, Npad64,
                Kpad64, ntab * noff, KCH, Npad, tab);
  }
  // split Wm rows
  const int64_t rows = Lv.nbox * R;
  char* wms = (char*)ctx_buf(ctx, "wms", (size_t)rows * 2 * KpadTC * F::EL + 64);
  FMMA_LAUNCH(ctx, k_split_wm<BF16>, grid_for(rows * KpadTC / (16 / F::EL), 256, (int64_t)ctx->sm_count * 32), 256, 0,
              Wm64, rows, P, Kpad64, KpadTC, wms);
  // The 2-SM kernel (256-row tiles over SM pairs) on levels with at least one
  // tile per cluster; smaller levels take the 1-SM kernel with its slot split.
  // Producer warps: 8 when two epilogue column groups hold a row's sums in at
  // most 3 chunks of 16 columns a thread (N <= 96), else 4 (three groups).
  // cp.async delivery grows with the warps that issue it (1 per SM sub-
  // partition carries ~12 B per SM cycle from L2, 2 carry ~22).
  const int nch = Npad / 16;
  const int npw = (nch + 1) / 2 <= 3 ? 8 : 4;
  const int cpt = npw == 8 ? (nch + 1) / 2 : (nch + 2) / 3;  // 16-column chunks per epilogue thread
#define FMMA_TC_VARIANT(CALL)                                          \
  do {                                                                 \
    if (npw == 8) {                                                    \
      if (cpt == 1) CALL(1, 8); else if (cpt == 2) CALL(2, 8);         \
      else CALL(3, 8);                                                 \
    } else {                                                           \
      if (cpt <= 3) CALL(3, 4); else if (cpt == 4) CALL(4, 4);         \
      else if (cpt == 5) CALL(5, 4); else CALL(6, 4);                  \
    }                                                                  \
  } while (0)

  // A pipeline stage holds `units` (slot, K chunk) units: one barrier wait and
  // one MMA commit per stage.  Each commit costs the tensor pipe a few hundred
  // cycles, as much as a unit's six MMAs at small P, so stages take 4 units
  // when a slot is one K chunk and 2 otherwise, keeping at least three stages
  // in flight (the C5 forest's M2L 23.3 -> 19.8 ms with 4; the C3 M2L 80 ->
  // 75 ms with 2).
  const size_t unit2_bytes = (size_t)2 * kTcM * F::ROW + (size_t)Npad * F::ROW;
  const size_t unit1_bytes = (size_t)2 * kTcM * F::ROW + (size_t)2 * Npad * F::ROW;
  const size_t smem_room = kTcSmemMax - 1024 - kTcStaticSmem;
  auto pick_units = [&](size_t unit_bytes) {
    const int asked = units_pref > 0 ? units_pref : ctx->tc_units;
    int u = asked > 0 ? std::min(asked, kTcMaxUnits) : (KCH == 1 ? 4 : 2);
    while (u > 1 && smem_room / (unit_bytes * u) < (asked > 0 ? 2u : 3u)) --u;
    return u;
  };
  const int units2 = pick_units(unit2_bytes);
  const size_t stage2_bytes = unit2_bytes * units2;
  const size_t smem2 = std::min<size_t>((size_t)kTcMaxStages, smem_room / stage2_bytes) * stage2_bytes + 1024;
  int ncl2 = -1;
  std::vector<int4> tiles;
  const int pair_want = pair_pref >= 0 ? pair_pref : (ctx->tc_pair != 0 ? 1 : 0);
  if (pair_want && Npad % 16 == 0) {
#define FMMA_TC2_CLUSTERS(C_, N_) ncl2 = tc2_max_clusters<BF16, C_, N_>(ctx, smem2)
    FMMA_TC_VARIANT(FMMA_TC2_CLUSTERS);
#undef FMMA_TC2_CLUSTERS
    if (ncl2 > 0) {
      tiles = m2l_tiles(Lv, R, kTc2M);
      if ((int)tiles.size() < ncl2) {
        ncl2 = -1;
        tiles.clear();
      }
    }
  }
  const bool pair = ncl2 > 0;
  // tiles and their non-empty slots
  if (!pair) tiles = m2l_tiles(Lv, R, kTcM);
  const int ntiles = (int)tiles.size();
  int4* dt = ctx_buf_t<int4>(ctx, "tc_tiles" + std::to_string(v), tiles.size());
  upload(ctx, dt, tiles.data(), sizeof(int4) * tiles.size());
  int* tnq = ctx_buf_t<int>(ctx, "tc_tnq", (size_t)ntiles);
  int* tq = ctx_buf_t<int>(ctx, "tc_tq", (size_t)ntiles * nfar);
  FMMA_LAUNCH(ctx, k_tile_slots, grid_for((int64_t)ntiles * 32, 256, (int64_t)ctx->sm_count * 16), 256, 0, dt, ntiles,
              Lv.slot_mask, nfar, R, tnq, tq);
  int* err = m2l_err_slot(ctx, v);
  FMMA_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));

  TcParams prm;
  prm.tiles = dt;
  prm.ntiles = ntiles;
  prm.tile_nq = tnq;
  prm.tile_q = tq;
  prm.il = Lv.il;
  prm.row_box = Lv.row_box;
  prm.slot_off = slot_off;
  prm.wms = wms;
  prm.tab = tab;
  prm.Wl = Wl64;
  prm.P = P;
  prm.Kpad64 = Kpad64;
  prm.KpadTC = KpadTC;
  prm.KCH = KCH;
  prm.Npad = Npad;
  prm.nfar = nfar;
  prm.R = R;
  prm.noff = noff;
  // Drain the accumulator after about kDrainSteps MMA accumulation steps (the
  // tensor core's FP32 sums round toward zero, so the error grows with the
  // steps summed in TMEM): 2 slots at P = 216 (7 K chunks x 2 steps x 3
  // products each), more slots for small P, whose slots are a single chunk
  // and would otherwise stall on the epilogue every few hundred cycles.
  const int steps_per_slot = KCH * F::NSTEP * 3;
  prm.group = ctx->tc_group > 0 ? std::min(ctx->tc_group, 189)
                                 : std::max(kGroupSlotsDefault, std::min(16, kDrainSteps / steps_per_slot));
  prm.a_reuse = 1;
  int cols = 32;
  while (cols < 2 * Npad) cols <<= 1;
  prm.tmem_cols = cols;
  prm.err = err;
  prm.wait_cycles = ctx->tc_wait_cycles > 0 ? ctx->tc_wait_cycles : kWaitCycles;
  prm.hold = nullptr;
  if (ctx->tc_hold) {  // test hook: a flag that nothing sets
    int* hold = ctx_buf_t<int>(ctx, "tc_hold", 1);
    FMMA_CHECK_CUDA(cudaMemsetAsync(hold, 0, sizeof(int), ctx->stream));
    prm.hold = hold;
  }
  prm.units = pair ? units2 : pick_units(unit1_bytes);
  const size_t stage_bytes = pair ? stage2_bytes : unit1_bytes * prm.units;
  const int stages_cap = ctx->tc_stages >= 2 ? std::min(ctx->tc_stages, kTcMaxStages) : kTcMaxStages;
  const int stages = (int)std::min<size_t>((size_t)stages_cap, smem_room / stage_bytes);
  FMMA_REQUIRE(stages >= 2, "tensor-core M2L: shared memory too small for two stages");
  prm.stages = stages;
  const size_t smem = (size_t)stages * stage_bytes + 1024;
  // Levels with fewer tiles than SMs split each tile's slot list into parts
  // run by different CTAs; their partial sums are added by k_tc_split_sum.
  // The plan autotuner may ask for none, half or twice as many parts.
  int nsplit = 1;
  if (!pair && ntiles < ctx->sm_count) {
    nsplit = std::min(16, std::max(1, (ctx->sm_count + ntiles - 1) / ntiles));
    const int lv = (size_t)v < ctx->m2l_split.size() ? ctx->m2l_split[(size_t)v] : 0;
    const int mode = lv != 0 ? lv : ctx->tc_split;
    if (mode == 1) nsplit = 1;
    else if (mode == 2) nsplit = std::max(1, nsplit / 2);
    else if (mode == 3) nsplit = std::min(16, 2 * nsplit);
  }
  prm.nsplit = nsplit;
  prm.part = nsplit > 1 ? ctx_buf_t<double>(ctx, "tc_part", (size_t)ntiles * nsplit * kTcM * Npad) : nullptr;
  const unsigned grid = (unsigned)std::min<int64_t>((int64_t)ntiles * nsplit, ctx->sm_count);
  kernel_timer_begin(ctx);
  if (pair) {
#define FMMA_TC2_LAUNCH(C_, N_) launch_tc2<BF16, C_, N_>(ctx, ncl2, smem, prm)
    FMMA_TC_VARIANT(FMMA_TC2_LAUNCH);
#undef FMMA_TC2_LAUNCH
  } else {
#define FMMA_TC_LAUNCH(C_, N_) launch_tc<BF16, C_, N_>(ctx, grid, smem, prm)
    FMMA_TC_VARIANT(FMMA_TC_LAUNCH);
#undef FMMA_TC_LAUNCH
  }
#undef FMMA_TC_VARIANT
  if (nsplit > 1)
    FMMA_LAUNCH(ctx, k_tc_split_sum, grid_for((int64_t)ntiles * kTcM * P, 256), 256, 0, dt, ntiles, nsplit, prm.part,
                Lv.row_box, R, Kpad64, P, Npad, Wl64);
  kernel_timer_end(ctx, 2.0 * P * P * R, v);
  ctx->m2l_err_flags.push_back(err);
}

void m2l_level_tc(fmma_ctx* ctx, bool bf16, int pair, int units, const Level& Lv, int v, int nfar, const int* slot_off,
                  int P,
                  int Kpad64, int R, const double* Wm64, double* Wl64, const double* tab64, int Npad64,
                  const std::string& tabkey, int noff, int ntab) {
  if (bf16)
    m2l_level_tc_t<true>(ctx, pair, units, Lv, v, nfar, slot_off, P, Kpad64, R, Wm64, Wl64, tab64, Npad64, tabkey, noff, ntab);
  else
    m2l_level_tc_t<false>(ctx, pair, units, Lv, v, nfar, slot_off, P, Kpad64, R, Wm64, Wl64, tab64, Npad64, tabkey, noff, ntab);
}

}  // namespace fmma_b200
