// fmma_internal.cuh — context, scratch buffers, launch accounting and the
// declarations shared by the .cu files of libfmma_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fmma_b200.h"

namespace fmma_b200 {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  fmma_status code;
  Error(fmma_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& m);

#define FMMA_CHECK_CUDA(expr)                                                        \
  do {                                                                               \
    cudaError_t e_ = (expr);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      throw ::fmma_b200::Error(e_ == cudaErrorMemoryAllocation ? FMMA_ERR_OOM        \
                                                               : FMMA_ERR_CUDA,      \
                               std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    }                                                                                \
  } while (0)

#define FMMA_REQUIRE(cond, msg)                                           \
  do {                                                                    \
    if (!(cond)) throw ::fmma_b200::Error(FMMA_ERR_INVALID_ARG, (msg));   \
  } while (0)

// ---------------------------------------------------------------------------
// problem geometry and tree
// ---------------------------------------------------------------------------
constexpr int kMaxDim = 3;
constexpr int kMaxNodes = 16;  // Chebyshev nodes per dimension

// Cube of src/fmm_core.cpp:160-173, computed on the device in the caller's
// coordinate type and kept in both precisions.
struct Cube {
  double origin[kMaxDim];
  double Len;
  float originf[kMaxDim];
  float Lenf;
  int nonfinite;  // a NaN/Inf coordinate was seen
  int pad;
};

// Keys: the problem id of a forest occupies the top 12 bits, the Morton code
// of the box at its level the low 52 bits (dim 0 most significant inside
// each d-bit group).  A single solve is a forest of one problem (id 0).
constexpr int kPidShift = 52;
constexpr int kMaxProblems = 4096;
constexpr uint64_t kMortonMask = (1ull << kPidShift) - 1ull;
__host__ __device__ inline int key_pid(uint64_t k) { return (int)(k >> kPidShift); }

// One virtual level of the forest of sparse uniform-depth trees.  Levels are
// counted from the leaves: at virtual level v a box of problem p sits at the
// real level depth[p] - 1 - v of the 2^l grid.  Boxes are the non-empty boxes
// (holding targets or sources), sorted by key, so a box's points are a
// contiguous range of the key-sorted point arrays and its children a
// contiguous range of level v - 1.
constexpr int kSlotWords = 6;  // 189 far slots as a bit set

struct Level {
  int v = 0;
  int64_t nbox = 0;
  uint64_t* key = nullptr;   // (problem, Morton) key
  int* tb = nullptr;         // target range [tb, te) in sorted target order
  int* te = nullptr;
  int* sb = nullptr;         // source range [sb, se) in sorted source order
  int* se = nullptr;
  int* cb = nullptr;         // children [cb, ce) at virtual level v - 1
  int* ce = nullptr;
  int* parent = nullptr;     // parent box at virtual level v + 1 (-1 at a root)
  // M2L rows: boxes holding targets at real level >= 2, grouped by
  // (problem, child-parity class); segs = (problem, class, row_begin, row_end)
  int64_t nrow = 0;
  int* row_box = nullptr;
  std::vector<int4> segs;
  int* il = nullptr;                   // [nrow][nfar] source box or -1
  unsigned* slot_mask = nullptr;       // [nrow][kSlotWords] bit q set when il[row][q] >= 0
  int64_t il_pairs = 0;                // number of (target box, source box) pairs
  // M2L operator tables of this level: one per problem with a real level >= 2
  std::vector<int> table_pid;          // table id -> problem
  std::vector<int> pid_table;          // problem -> table id or -1
};

struct Tree {
  int dim = 0;
  int vmax = 0;                // deepest problem's Depth
  int nprob = 0;
  std::vector<int> depth;      // Depth of each problem
  int* d_depth = nullptr;
  std::vector<Cube> h_cube;    // cube of each problem
  Cube* d_cube = nullptr;
  int64_t nt = 0, ns = 0;
  int* perm_t = nullptr;       // sorted target -> original index
  int* perm_s = nullptr;       // sorted source -> original index
  std::vector<Level> lev;      // virtual levels 0 (leaves) .. vmax-1
  // near lists at the leaves: [nnear_rows][3^d] source box or -1
  int64_t nnear_rows = 0;
  int* near_row_box = nullptr;
  int* near = nullptr;
  int64_t p2p_pairs = 0;
  // counted from the sorted keys before the levels are emitted: M2L rows of
  // every virtual level and near-field rows; a nonzero *d_err means a level
  // emitted more boxes than counted (checked at the last read-back)
  std::vector<int> row_count;
  int64_t near_count = 0;
  int* d_err = nullptr;
  // the pair counts (il_pairs per level, p2p_pairs) and d_err stay on the
  // device until the host needs them (tree_read_pairs), so the build itself
  // ends without a wait
  unsigned long long* d_pairs = nullptr;
  bool pairs_read = true;
  bool valid = false;
  // single-problem helpers
  int depth0() const { return depth.empty() ? 0 : depth[0]; }
  const Cube& cube0() const { return h_cube[0]; }
  // virtual level of real level l for a single problem
  Level& real(int l) { return lev[(size_t)(depth[0] - 1 - l)]; }
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

enum Stage { ST_TREE = 0, ST_P2M, ST_M2M, ST_M2L, ST_L2L, ST_L2P, ST_P2P, ST_EXACT, ST_TOTAL };

}  // namespace fmma_b200

// pipeline-stage unit counts the plan autotuner tries for the tensor-core M2L
constexpr int kM2LUnitChoices[3] = {1, 2, 4};
constexpr int kM2LEngines = 1 + 2 * 3;  // FP64 + tensor-core (1-SM, 2-SM) x unit choices

struct fmma_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int kernel_id = FMMA_KERNEL_INV_R;
  double p0 = 0.0;
  std::map<std::string, fmma_b200::DevBuf> bufs;   // grow-only scratch
  std::map<std::string, fmma_b200::DevBuf> ops;    // cached operator tables
  // device allocator of bufs and ops (null: cudaMalloc / cudaFree)
  fmma_alloc_fn alloc_fn = nullptr;
  fmma_free_fn free_fn = nullptr;
  void* alloc_user = nullptr;
  cudaEvent_t ev[2 * FMMA_NUM_STAGES] = {};
  bool ev_used[FMMA_NUM_STAGES] = {};
  double stage_ms[FMMA_NUM_STAGES] = {};
  int64_t launches = 0;
  fmma_b200::Tree tree;
  int sm_count = 148;
  void* pinned = nullptr;  // small pinned staging buffer for readbacks
  size_t pinned_bytes = 0;
  char* up_host = nullptr;  // pinned upload arena: copies in flight use [0, up_used)
  size_t up_cap = 0, up_used = 0;
  // per-launch timing of the dominant (M2L) kernel of the last solve
  static constexpr int kMaxTimed = 64;
  cudaEvent_t kev[2 * kMaxTimed] = {};
  double kflops[kMaxTimed] = {};
  int ktag[kMaxTimed] = {};    // virtual level of each timed launch
  double kms[kMaxTimed] = {};  // its duration after stages_collect
  int ktimed = 0;
  double m2l_kernel_ms = 0.0, m2l_flops = 0.0;
  int64_t m2l_launches = 0;
  std::vector<int*> m2l_err_flags;  // device flags of bounded waits, checked at the end
  // bound of the tensor-core M2L's pipeline waits in SM clocks (0: ~2 s) and
  // the test hook that makes its MMA issuer wait for a flag nothing sets
  long long tc_wait_cycles = 0;
  bool tc_hold = false;
  // tensor-core M2L options (fmma_set_m2l_options): the 2-SM kernel on levels
  // with a tile per cluster (-1 default = on, 0 off), the pipeline depth cap
  // (0: as many stages as fit, up to 8), the slots per accumulator drain
  // (0: about 84 MMA accumulation steps) and the (slot, K chunk) units per
  // pipeline stage (0: by the operand size)
  int tc_pair = -1;
  int tc_stages = 0;
  int tc_group = 0;
  int tc_units = 0;
  // stream capture of a sweep (a plan's CUDA graph): uploads of constant data
  // and event timers are skipped, the device buffers keep the warm-up's data
  bool capturing = false;
  // per virtual level M2L engine chosen by the autotuner: -1 the context's
  // options, 0 the FP64 DMMA kernel, 1 + 2 * i + pair the tensor-core kernel
  // (pair 0: 1-SM, 1: 2-SM) with kM2LUnitChoices[i] units per stage
  std::vector<int> m2l_engine;
  // slot split of the 1-SM tensor-core M2L on levels with fewer tiles than
  // SMs: 0 enough parts to fill the SMs, 1 no split, 2 half as many parts,
  // 3 twice as many (at most 16); per virtual level (the autotuner's choice,
  // 0 = tc_split) and for the context (fmma_set_schedule_options)
  std::vector<int> m2l_split;
  int tc_split = 0;
  // leaf evaluation (L2P): 0 by the targets per leaf, 1 lanes over targets,
  // 2 lanes over coefficients (with one rhs the leaf L2L fused in)
  int l2p_mode = 0;
  std::map<std::string, int> tuner;  // decisions by workload key
  std::string tuner_path;            // optional file the tuner cache persists to
  // user device functor (kernel_id == kUserKernel)
  fmma_user_hook user_hook = nullptr;
  void* user_ptr = nullptr;
  std::shared_ptr<void> user_own;  // keeps a library-owned hook state (expression kernels) alive
  int user_ti = 1;
  int user_gen = 0;
};

namespace fmma_b200 {

constexpr int kUserKernel = 1000;  // kernel_id of a user functor installed through a hook

inline bool ctx_translation_invariant(const fmma_ctx* ctx) {
  return ctx->kernel_id == kUserKernel ? ctx->user_ti != 0 : ctx->kernel_id != FMMA_KERNEL_SUM2_OVER_R2;
}

// Installs a kernel given as an expression, compiled at run time (jit.cu).
void set_kernel_expr(fmma_ctx* ctx, const char* expr, int translation_invariant);

// Calls the user hook; throws on a non-zero cudaError_t.
inline void call_user_hook(fmma_ctx* ctx, fmma_user_launch& a) {
  a.stream = (void*)ctx->stream;
  int e = ctx->user_hook(&a, ctx->user_ptr);
  ctx->launches++;
  if (e == (int)cudaErrorInvalidSource) throw Error(FMMA_ERR_INVALID_ARG, "kernel expression failed to compile");
  if (e != 0) throw Error(FMMA_ERR_CUDA, "user kernel hook failed with CUDA error " + std::to_string(e));
}

// Device scratch owned by the context, reused across calls, grown on demand.
// Device memory through the context's allocator (cudaMalloc / cudaFree by
// default): dev_alloc returns null when the allocation fails; dev_free is
// called with the stream idle.
void* dev_alloc(fmma_ctx* ctx, size_t bytes);
void dev_free(fmma_ctx* ctx, void* p, size_t bytes);
// Releases every scratch buffer and cached operator (stream synchronised).
void release_device_memory(fmma_ctx* ctx);
void* ctx_buf(fmma_ctx* ctx, const std::string& name, size_t bytes);
template <typename T>
T* ctx_buf_t(fmma_ctx* ctx, const std::string& name, size_t count) {
  return static_cast<T*>(ctx_buf(ctx, name, count * sizeof(T) + 16));
}
// Pinned host scratch (readback of small results).
void* ctx_pinned(fmma_ctx* ctx, size_t bytes);
// Host -> device copy of constant data of a sweep; skipped while a sweep is
// being captured (the buffer already holds the same data).
// Host -> device copy of small host-built arrays (tile lists, tables),
// staged through the context's pinned upload arena so that the copy is
// asynchronous (a copy from pageable memory may make the driver wait for the
// stream first).  Skipped while a sweep is being captured.
void upload(fmma_ctx* ctx, void* dst, const void* src, size_t bytes);

inline void after_launch(fmma_ctx* ctx) {
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error(FMMA_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

#define FMMA_LAUNCH(ctx, kern, grid, block, smem, ...)                       \
  do {                                                                       \
    kern<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);           \
    ::fmma_b200::after_launch(ctx);                                          \
  } while (0)

inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// CUDA-event timing of individual M2L kernel launches (algorithmic flops).
void kernel_timer_begin(fmma_ctx* ctx);
// M2L launch timer; flops_per_pair x the level's (target box, source box)
// pairs (read when the timers are collected) gives the launch's flops
void kernel_timer_end(fmma_ctx* ctx, double flops_per_pair, int tag);
// brings the tree's pair counts to the host (one wait, once per build) and
// checks the build's overflow flag
void tree_read_pairs(fmma_ctx* ctx);

// Stage timing with CUDA events on the context stream.
void stage_begin(fmma_ctx* ctx, Stage s);
void stage_end(fmma_ctx* ctx, Stage s);
void stages_reset(fmma_ctx* ctx);
void stages_collect(fmma_ctx* ctx);

// ---------------------------------------------------------------------------
// primitives (prims.cu)
// ---------------------------------------------------------------------------
// Exclusive scan of n int32 values; writes the total to *total_dev (device).
void scan_exclusive(fmma_ctx* ctx, const int* in, int* out, int64_t n, int* total_dev);
// Stable LSD radix sort of (key, val) pairs on bits [bit0, bit1) of the key.
// Results end in keys/vals (tmp buffers from the context).
void radix_sort_pairs(fmma_ctx* ctx, uint64_t* keys, int* vals, int64_t n, int bit0, int bit1);
// Copy n ints device -> host (synchronous on the context stream).
void read_ints(fmma_ctx* ctx, const int* dev, int* host, int n);
// error flag of the tensor-core M2L at virtual level v (one buffer for all
// levels), and the check of a solve's flags with one read (FMMA_ERR_TIMEOUT)
int* m2l_err_slot(fmma_ctx* ctx, int v);
void check_m2l_errs(fmma_ctx* ctx, const std::vector<int*>& flags);

// ---------------------------------------------------------------------------
// tree (tree.cu)
// ---------------------------------------------------------------------------
// Builds ctx->tree for a forest: points of problem p are tgt[toff[p]..toff[p+1])
// and src[soff[p]..soff[p+1]] (host offsets, device coordinates), depth[p] its
// Depth.  When `lists` is false only the leaves and permutations are built.
template <typename T>
void build_forest(fmma_ctx* ctx, int dim, const std::vector<int64_t>& toff, const T* tgt,
                  const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth, bool lists);

// Single problem: a forest of one.
template <typename T>
void build_tree(fmma_ctx* ctx, int dim, int depth, int64_t nt, const T* tgt, int64_t ns, const T* src, bool lists);

// Largest leaf occupancy at `depth` (targets, sources) of every problem.
template <typename T>
void leaf_occupancy(fmma_ctx* ctx, int dim, const std::vector<int64_t>& toff, const T* tgt,
                    const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth,
                    std::vector<int>* max_t, std::vector<int>* max_s);

// Row-major leaf index (reference numbering) of every point, one problem.
template <typename T>
void export_bins(fmma_ctx* ctx, int dim, int depth, int64_t nt, const T* tgt, int64_t ns,
                 const T* src, int64_t* tbox_dev, int64_t* sbox_dev, Cube* cube_out);

// Global Chebyshev approximation (cheb.cu): coefficients of nfunc functions
// from their values at the tensor nodes, and evaluation at points (device
// pointers; values and coef must not alias).
void cheb_fit(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* values, double* coef);
void cheb_eval(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* coef, int64_t npts, const double* pts,
               double* out);

// Bounding cube of one problem (src/fmm_core.cpp:158-173) into the context
// buffer `cube_buf`; returns the device copy and fills *host.
template <typename T>
const Cube* problem_cube(fmma_ctx* ctx, int dim, int64_t nt, const T* tgt, int64_t ns, const T* src,
                         const char* cube_buf, Cube* host);

// Morton helpers (host + device).  Level bit b of coordinate q sits at key
// bit b * dim + (dim - 1 - q).  Bits are spread and gathered with the usual
// shift-and-mask sequences, in constant time.
__host__ __device__ inline uint64_t morton_spread2(uint64_t x) {  // bit i -> bit 2i
  x &= 0xffffffffull;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}
__host__ __device__ inline uint64_t morton_gather2(uint64_t x) {  // bit 2i -> bit i
  x &= 0x5555555555555555ull;
  x = (x | (x >> 1)) & 0x3333333333333333ull;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffull;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffull;
  x = (x | (x >> 16)) & 0x00000000ffffffffull;
  return x;
}
__host__ __device__ inline uint64_t morton_spread3(uint64_t x) {  // bit i -> bit 3i (i < 21)
  x &= 0x1fffffull;
  x = (x | (x << 32)) & 0x001f00000000ffffull;
  x = (x | (x << 16)) & 0x001f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
__host__ __device__ inline uint64_t morton_gather3(uint64_t x) {  // bit 3i -> bit i
  x &= 0x1249249249249249ull;
  x = (x | (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x | (x >> 4)) & 0x100f00f00f00f00full;
  x = (x | (x >> 8)) & 0x001f0000ff0000ffull;
  x = (x | (x >> 16)) & 0x001f00000000ffffull;
  x = (x | (x >> 32)) & 0x00000000001fffffull;
  return x;
}
__host__ __device__ inline uint64_t morton_encode(const int* c, int dim, int bits) {
  const uint64_t m = bits >= 32 ? 0xffffffffull : ((1ull << bits) - 1ull);
  if (dim == 3)
    return (morton_spread3((uint64_t)c[0] & m) << 2) | (morton_spread3((uint64_t)c[1] & m) << 1) |
           morton_spread3((uint64_t)c[2] & m);
  if (dim == 2) return (morton_spread2((uint64_t)c[0] & m) << 1) | morton_spread2((uint64_t)c[1] & m);
  return (uint64_t)c[0] & m;
}
__host__ __device__ inline void morton_decode(uint64_t k, int dim, int bits, int* c) {
  const int nb = bits * dim;
  if (nb < 64) k &= (1ull << nb) - 1ull;
  if (dim == 3) {
    c[0] = (int)morton_gather3(k >> 2);
    c[1] = (int)morton_gather3(k >> 1);
    c[2] = (int)morton_gather3(k);
  } else if (dim == 2) {
    c[0] = (int)morton_gather2(k >> 1);
    c[1] = (int)morton_gather2(k);
  } else {
    c[0] = (int)k;
  }
}

// Far-slot tables per child-parity class: slot q of class c is the block
// position j (base-6 digits, last dimension fastest) and the far-offset id
// (index among the 7^d - 3^d offsets with |o|_inf > 1, row-major in o+3).
struct FarTables {
  int nfar = 0, noff = 0, nclass = 0;
  int slot_j[8][189];
  int slot_off[8][189];
  int off_vec[316][3];
  int jslot[8][216];  // [class][position in the 6^d window] -> slot, -1 for the near boxes
};
const FarTables& far_tables(int dim);

// warp-per-box stage kernels (fmm_warp.cu)
void launch_p2m_warp(fmma_ctx* ctx, const Level& Lf, const double* sx, int64_t ns, const double* ws, int R,
                     const Cube* cubes, const int* depth, int d, bool isf, int n, int P, int Kpad, const double* Tn,
                     double* Wm, int grid_n = 0);
void launch_l2p_warp(fmma_ctx* ctx, const Level& Lf, const double* tx, int64_t nt, const Cube* cubes,
                     const int* depth, int d, bool isf, int n, int P, int Kpad, int R, const double* Tn,
                     const double* Wl, double* pot, int ostride, int ooff);
void launch_m2m_warp(fmma_ctx* ctx, const Level& C, const Level& Pl, int vpar, const int* depth, int d, int n, int P,
                     int Kpad, int R, const double* A, const double* Wc, double* Wp);
void launch_l2l_warp(fmma_ctx* ctx, const Level& C, int vchild, const int* depth, int d, int n, int P, int Kpad, int R,
                     const double* A, const double* Wp, double* Wc);
// Leaf L2L fused into L2P for one right-hand side on leaves with few targets
// (pot[t] written for every target of the leaf rows); false when the case is
// not covered (dense leaves, other node counts): run L2L and L2P instead.
// mode: the context's l2p_mode (0 by the targets per leaf, 1 lanes over
// targets, 2 lanes over coefficients)
bool l2p_coef_lanes(const Level& Lf, int64_t nt, int mode);
bool l2lp_leaf_ok(const Level& Lf, int64_t nt, int d, int n, int mode);
bool launch_l2lp_leaf(fmma_ctx* ctx, const Level& Lf, const double* tx, int64_t nt, const Cube* cubes,
                      const int* depth, int d, bool isf, int n, int Kpad, const double* Tn, const double* A,
                      const double* Wp, const double* Wc, double* pot);
// Neighbour lists of every box of level Lv (nbr, [nbox][3^d]) from the
// parent level's (pnbr; Pl == nullptr at the top level), and the far lists
// (il, slot_mask) of Lv's rows; row_of_box is scratch of Lv.nbox ints.
void launch_lists_topdown(fmma_ctx* ctx, const Level& Lv, const Level* Pl, const int* pnbr, int d, int nfar,
                          const int* jslot, int* nbr, int* row_of_box, unsigned long long* pairs);
// P2P near lists of the leaf rows from the leaf neighbour lists.
void launch_near_rows(fmma_ctx* ctx, const int* nbr, const int* row_box, int64_t nrow, int d, const int* sb,
                      const int* se, int* near);

// ---------------------------------------------------------------------------
// FMM stages
// ---------------------------------------------------------------------------
struct ChebTables {
  int n = 0;                  // nodes per dimension
  double node[kMaxNodes];     // cos((2k+1)pi/(2n)), descending
  double Tn[kMaxNodes * kMaxNodes];      // Tn[k*n+j] = T_j(node_k)
  double A[2][kMaxNodes * kMaxNodes];    // M2M 1-D operators, s = -1, +1:
                                         // A[s][i*n+j] = S_n(node_i, (node_j+s)/2)
};
ChebTables make_cheb_tables(int n);

struct SolveArgs {
  int dim, n, P, depth, trans_sym, precision, nrhs;
  int kernel_id;
  double p0;
  int tree = 0;  // the tree solver: M2P per level instead of M2L/L2L/L2P
};

}  // namespace fmma_b200
