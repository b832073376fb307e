/*
 * fmma_b200.h — C ABI of the B200 (sm_100a) implementation of FMMA's `exact`
 * and `fmm` solvers.
 *
 * Every entry point takes plain pointers and sizes.  Point arrays are
 * array-of-structs `[n][dim]` (the memory image of the reference's
 * `std::vector<std::array<T,DIM>>`), weights are `[nrhs][n_src]`, results are
 * `[nrhs][n_tgt]`.  `mem_kind` says whether the pointers are host or device
 * memory; host buffers are staged through the context's pinned buffers.
 * The library never frees caller memory.  A context (`fmma_ctx`) owns one
 * CUDA stream, its device scratch and its operator-table cache; it is not
 * thread-safe (same contract as the reference object, which keeps a sticky
 * `Depth` and a mutable time log).
 *
 * Errors are returned as `fmma_status`; `fmma_last_error()` gives the message
 * of the last failure on the calling thread.  No entry point calls exit().
 */
#ifndef FMMA_B200_H
#define FMMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fmma_status {
  FMMA_OK = 0,
  FMMA_ERR_INVALID_ARG = 1,       /* sizes, NaN/Inf coordinates, bad ids    */
  FMMA_ERR_UNSUPPORTED_SOLVER = 2,/* unknown solver names                   */
  FMMA_ERR_OOM = 3,               /* device allocation failed               */
  FMMA_ERR_CUDA = 4,              /* a CUDA runtime call failed             */
  FMMA_ERR_TIMEOUT = 5,           /* a bounded device wait gave up          */
  FMMA_ERR_NO_DEVICE = 6          /* no CUDA device / extension not usable  */
} fmma_status;

/* Built-in interaction kernels f(x, y).  Ids are shared with the CPU oracle.
 * "0 at coincidence" means f(x, x) = 0 exactly (the singular kernels skip
 * the self term).                                                           */
typedef enum fmma_kernel_id {
  FMMA_KERNEL_INV_R = 0,         /* 1/|x-y|, no guard: the reference default
                                    functor (include/fmma/fmma.hpp:55-63)     */
  FMMA_KERNEL_INV_R_SAFE = 1,    /* 1/|x-y|, 0 at coincidence                */
  FMMA_KERNEL_INV_DIFF = 2,      /* 1/(x-y), 1D only, 0 at coincidence       */
  FMMA_KERNEL_LOG_R = 3,         /* log|x-y|, 0 at coincidence               */
  FMMA_KERNEL_GAUSSIAN = 4,      /* exp(-|x-y|^2 / p0)                       */
  FMMA_KERNEL_MULTIQUADRIC = 5,  /* sqrt(|x-y|^2 + p0)                       */
  FMMA_KERNEL_SUM_OVER_R2 = 6,   /* sum_d (x-y)_d / |x-y|^2  (reference test
                                    kernel, test/src/fmma/fmm.cpp:82-91)     */
  FMMA_KERNEL_SUM2_OVER_R2 = 7,  /* |x+y|^2 / |x-y|^2: NOT translation
                                    invariant (test/src/fmma/fmm.cpp:151-160) */
  FMMA_KERNEL_COUNT = 8
} fmma_kernel_id;

typedef enum fmma_solver {
  FMMA_SOLVER_EXACT = 0,   /* src/fmma.cpp:80-101  */
  FMMA_SOLVER_FMM = 1,     /* src/fmm.cpp:15-144   */
  FMMA_SOLVER_TREE = 2,    /* src/tree.cpp:12-100: P2M, M2M, M2P per level, P2P; FP64, built-in kernels */
  FMMA_SOLVER_NRNMM = 3    /* src/nrnmm.cpp:13-102: one grid of nrn_N^dim boxes, P2M, M2P from every
                              box not adjacent to the target's, P2P from the adjacent ones; FP64.
                              The `depth` argument of a solve carries nrn_N (<= 0: the default
                              (int)(sqrt(3) * n_src^(1/(2 dim))) + 1), *depth_used returns it. */
} fmma_solver;

typedef enum fmma_precision {
  FMMA_PREC_FP64 = 0,          /* plain: FP64 everywhere                      */
  FMMA_PREC_MIXED_TF32X3 = 1,  /* FP32 compensated P2P, TF32x3 tcgen05 M2L    */
  FMMA_PREC_MIXED_BF16X3 = 2   /* FP32 compensated P2P, BF16x3 tcgen05 M2L    */
} fmma_precision;

typedef enum fmma_mem_kind {
  FMMA_MEM_HOST = 0,
  FMMA_MEM_DEVICE = 1
} fmma_mem_kind;

typedef struct fmma_ctx fmma_ctx;

/* ---- context ------------------------------------------------------------ */

/* Creates a context on CUDA device `device` (its own non-blocking stream). */
fmma_status fmma_ctx_create(int device, fmma_ctx** out);
fmma_status fmma_ctx_destroy(fmma_ctx* ctx);
/* Message of the last failure on this thread ("" if none). */
const char* fmma_last_error(void);
/* Library version string. */
const char* fmma_version(void);

/* Selects the interaction kernel; replaces fmma::FMMA::set_fn for built-in
 * functors (include/fmma/fmma.hpp:65-87).  `p0` is the kernel parameter
 * (Gaussian width^2, multiquadric shift), ignored by the other kernels.     */
fmma_status fmma_set_kernel(fmma_ctx* ctx, int kernel_id, double p0);

/* Default Depth of the reference: (int)(ln(n_tgt)/dim)+1, at least 1
 * (src/fmm.cpp:23-28).                                                      */
int fmma_default_depth(int64_t n_tgt, int dim);

/* ---- solve --------------------------------------------------------------
 * Replaces FMMA<T,DIM>::solve (src/fmma.cpp:143-207) for solvers "exact",
 * "fmm", "tree" and "nrnmm".  poly_ord = Chebyshev nodes per dimension - 1
 * (the reference's set_poly_ord), depth <= 0 selects the reference default
 * (for nrnmm, depth is nrn_N, the reference's set_nrn_N), trans_sym is the
 * reference's trans_sym_flag.  w == NULL means unit weights (the reference's
 * three-argument solve).  On return *depth_used (if not NULL) holds the
 * depth actually used, so a caller can keep the reference's sticky Depth.  */
fmma_status fmma_solve_d(fmma_ctx* ctx, int dim, int solver, int poly_ord,
                         int depth, int trans_sym, int precision,
                         int64_t n_tgt, const double* tgt,
                         int64_t n_src, const double* src,
                         int nrhs, const double* w, double* ans,
                         int mem_kind, int* depth_used);
/* float instantiation (FMMA<float,DIM>): box binning in float exactly as the
 * reference's float build does it; arithmetic in FP64; results rounded.    */
fmma_status fmma_solve_f(fmma_ctx* ctx, int dim, int solver, int poly_ord,
                         int depth, int trans_sym, int precision,
                         int64_t n_tgt, const float* tgt,
                         int64_t n_src, const float* src,
                         int nrhs, const float* w, float* ans,
                         int mem_kind, int* depth_used);

/* Per-dimension spellings of the two calls above. */
fmma_status fmma_solve_d1(fmma_ctx*, int, int, int, int, int, int64_t, const double*, int64_t, const double*, int, const double*, double*, int, int*);
fmma_status fmma_solve_d2(fmma_ctx*, int, int, int, int, int, int64_t, const double*, int64_t, const double*, int, const double*, double*, int, int*);
fmma_status fmma_solve_d3(fmma_ctx*, int, int, int, int, int, int64_t, const double*, int64_t, const double*, int, const double*, double*, int, int*);
fmma_status fmma_solve_f1(fmma_ctx*, int, int, int, int, int, int64_t, const float*, int64_t, const float*, int, const float*, float*, int, int*);
fmma_status fmma_solve_f2(fmma_ctx*, int, int, int, int, int, int64_t, const float*, int64_t, const float*, int, const float*, float*, int, int*);
fmma_status fmma_solve_f3(fmma_ctx*, int, int, int, int, int, int64_t, const float*, int64_t, const float*, int, const float*, float*, int, int*);

/* Exact sum at a subset of targets (the FP64 GPU oracle for large
 * configurations): ans[r][i] = sum_j w[r][j] f(tgt[rows[i]], src[j]).
 * Same kernel evaluation as the exact solver (src/fmma.cpp:80-101).        */
fmma_status fmma_exact_rows_d(fmma_ctx* ctx, int dim, int64_t nrows, const int64_t* rows,
                              int64_t n_tgt, const double* tgt, int64_t n_src,
                              const double* src, int nrhs, const double* w,
                              double* ans, int mem_kind);

/* Potential and its gradient with respect to the target position (the
 * adjoint's building block): grad[r][i][q] = d/dx_q of the computed c_i.
 * fmm: the exact derivative of the FMM's own result while each target stays
 * in its leaf: the far field differentiates the L2P interpolant (d S_n/d x),
 * the near field uses grad f; exact: direct sum of grad f.  ans may be NULL.
 * FP64 and built-in translation-invariant kernels only.  No counterpart in
 * the reference (it has no derivatives); the sums are src/fmm.cpp:113-141.  */
fmma_status fmma_solve_grad_d(fmma_ctx* ctx, int dim, int solver, int poly_ord,
                              int depth, int trans_sym, int precision,
                              int64_t n_tgt, const double* tgt,
                              int64_t n_src, const double* src,
                              int nrhs, const double* w, double* ans, double* grad,
                              int mem_kind, int* depth_used);

/* ---- forests of independent problems ---------------------------------------
 * nprob problems in one sweep: problem p owns the targets tgt[toff[p] ..
 * toff[p+1]) and sources src[soff[p] .. soff[p+1]) (host offset arrays of
 * nprob + 1 entries, concatenated point arrays), its own cube and Depth
 * depths[p].  Weights are [nrhs][soff[nprob]], results [nrhs][toff[nprob]].
 * Every stage runs once for all problems (levels are aligned at the leaves).
 * Same result per problem as fmma_solve_d on that problem alone.  No
 * counterpart in the reference (one problem per FMMA::solve call,
 * src/fmma.cpp:143-207); built-in kernels only.                            */
fmma_status fmma_forest_solve_d(fmma_ctx* ctx, int dim, int nprob,
                                const int64_t* toff, const double* tgt,
                                const int64_t* soff, const double* src,
                                int nrhs, const double* w, double* ans,
                                int poly_ord, const int* depths, int trans_sym,
                                int precision, int mem_kind);
/* Smallest Depth per problem whose largest leaf holds at most leaf_cap
 * targets and at most leaf_cap sources.                                     */
fmma_status fmma_forest_depths_d(fmma_ctx* ctx, int dim, int nprob,
                                 const int64_t* toff, const double* tgt,
                                 const int64_t* soff, const double* src,
                                 int leaf_cap, int mem_kind, int* depths);

/* ---- plans: one geometry, many weight sets --------------------------------
 * Builds the tree, lists, operator tables and buffers of a forest geometry
 * once (nprob = 1 for a single problem), picks per level the faster M2L engine
 * when `autotune` is set (tensor-core split precision or FP64 DMMA, timed on
 * this geometry; decisions kept in the context's tuner cache), and captures
 * the sweep P2M..P2P into a CUDA graph.  fmma_plan_execute_d replays it for
 * new weights [nrhs][n_src] (results [nrhs][n_tgt]).  The plan owns a private
 * context created on the parent's device with the parent's kernel.  No
 * counterpart in the reference (which rebuilds everything per solve).       */
typedef struct fmma_plan fmma_plan;
fmma_status fmma_plan_create_d(fmma_ctx* parent, int dim, int nprob,
                               const int64_t* toff, const double* tgt,
                               const int64_t* soff, const double* src,
                               int nrhs, int poly_ord, const int* depths,
                               int trans_sym, int precision, int autotune,
                               int mem_kind, fmma_plan** out);
fmma_status fmma_plan_execute_d(fmma_plan* plan, const double* w, double* ans,
                                int mem_kind);
/* Build time, last execution time (ms, CUDA events), levels run on each M2L
 * engine, nodes of the captured graph.                                      */
fmma_status fmma_plan_stats(fmma_plan* plan, double* build_ms, double* last_exec_ms,
                            int* levels_tc, int* levels_f64, int64_t* graph_nodes);
fmma_status fmma_plan_destroy(fmma_plan* plan);
/* Loads (and later saves) the autotuner's decisions from/to a text file.    */
fmma_status fmma_set_tuner_cache(fmma_ctx* ctx, const char* path);

/* ---- tree inspection (bit-exactness against the reference) ---------------
 * Bins targets and sources exactly like src/fmm_core.cpp:258-267 and
 * src/fmm.cpp:126-131 on the cube of src/fmm_core.cpp:160-173.  Writes the
 * reference's row-major leaf index of every point (dim 0 most significant,
 * src/fmm_core.cpp:204-212) and origin[dim], Len into origin_len[dim+1].    */
fmma_status fmma_tree_export_d(fmma_ctx* ctx, int dim, int depth,
                               int64_t n_tgt, const double* tgt,
                               int64_t n_src, const double* src,
                               int64_t* tgt_box, int64_t* src_box,
                               double* origin_len, int mem_kind);

/* After a solve with solver FMM: the far interaction list (M2L) of the
 * target box with row-major index `box` at `level` (grid 2^level per side),
 * restricted to boxes that hold sources, in the reference's lexicographic
 * order (src/fmm_core.cpp:15-63).  Returns the count in *count (<= 189). */
fmma_status fmma_interaction_list(fmma_ctx* ctx, int level, int64_t box,
                                  int64_t* out, int cap, int* count);
/* Same for the near list (P2P, src/fmm_core.cpp:79-115), leaf level.       */
fmma_status fmma_near_list(fmma_ctx* ctx, int64_t box,
                           int64_t* out, int cap, int* count);

/* Largest number of targets and of sources in one leaf at `depth`
 * (used to pick the depth for a leaf cap).                                 */
fmma_status fmma_max_leaf_occupancy_d(fmma_ctx* ctx, int dim, int depth,
                                      int64_t n_tgt, const double* tgt,
                                      int64_t n_src, const double* src,
                                      int mem_kind, int64_t* max_tgt,
                                      int64_t* max_src);

/* ---- device memory -----------------------------------------------------
 * The allocator of the context's device scratch and operator cache (and of
 * the private contexts of plans made from it afterwards).  No counterpart in
 * the reference, which keeps everything in host vectors.  For callers whose
 * device memory is owned by another allocator (a framework's caching
 * allocator, a memory pool with a budget).
 * alloc(bytes, stream, user) returns device memory usable on `stream` (the
 * context's stream), aligned to at least 256 bytes, or NULL when it cannot
 * serve the request: the call in progress then fails with FMMA_ERR_OOM and
 * the context stays usable.  A misaligned block is given back and the call
 * fails with FMMA_ERR_INVALID_ARG before any kernel uses it.
 * free(ptr, bytes, stream, user) gets back a pointer with the byte count
 * alloc was asked for, after `stream` has been synchronised.  Both run on
 * the calling host thread.  alloc = NULL restores cudaMalloc / cudaFree.
 * Switching allocators releases the context's scratch and cached operators
 * through the previous one; plans already made keep theirs (its functions
 * must stay valid until those plans are destroyed).                       */
typedef void* (*fmma_alloc_fn)(size_t bytes, void* stream, void* user);
typedef void (*fmma_free_fn)(void* ptr, size_t bytes, void* stream, void* user);
fmma_status fmma_set_allocator(fmma_ctx* ctx, fmma_alloc_fn alloc,
                               fmma_free_fn free_fn, void* user);

/* ---- tensor-core M2L options -------------------------------------------
 * Tuning switches of the mixed-precision M2L kernels; no counterpart in the
 * reference.  pair: the 2-SM kernel (a cluster of two CTAs on an SM pair,
 * M = 256 rows per tile) on levels with at least one 256-row tile per
 * cluster: -1 default (on), 0 off, 1 on.  stages: cap of the pipeline depth
 * (2..8; 0 = as many as shared memory holds).  group: far slots summed in
 * TMEM between two drains into FP32 registers (1..189; 0 = the default of
 * about 84 MMA accumulation steps, 2 slots at 6 nodes per dimension in 3-D).
 * units: (slot, K chunk) units per pipeline stage, i.e. per barrier wait and
 * MMA commit (1..4; 0 = by the operand size: several for small expansions,
 * whose units are a few MMAs each).  Results depend on group (FP32 rounding
 * of the partial sums) but not on pair, stages or units.  Plans made
 * afterwards inherit the options.                                          */
fmma_status fmma_set_m2l_options(fmma_ctx* ctx, int pair, int stages,
                                 int group, int units);

/* ---- schedule options ---------------------------------------------------
 * The choices the plan autotuner makes, set by hand for a context; no
 * counterpart in the reference.  m2l_split: how the 1-SM tensor-core M2L
 * splits the slot lists of levels with fewer 128-row tiles than SMs over
 * CTAs: 0 enough parts to fill the SMs (default), 1 none, 2 half as many,
 * 3 twice as many (at most 16); results move by FP32 rounding.  l2p_mode:
 * the leaf evaluation, 0 by the targets per leaf (default: lanes over
 * coefficients below 16 targets per leaf, with one rhs the leaf L2L fused
 * in), 1 lanes over targets, 2 lanes over coefficients; results move by
 * FP64 rounding.  Plans made afterwards inherit the options unless their
 * autotuner (mixed precision) picks its own.                               */
fmma_status fmma_set_schedule_options(fmma_ctx* ctx, int m2l_split, int l2p_mode);

/* ---- failure detection (tests) ------------------------------------------
 * Every pipeline wait of the tensor-core M2L is bounded; a wait that gives
 * up makes the solve return FMMA_ERR_TIMEOUT after the kernel has drained
 * (no copy or MMA left in flight, TMEM freed), and the context stays usable.
 * No counterpart in the reference (no device code).  This hook sets the
 * bound to wait_cycles SM clocks (<= 0: the default, about 2 s) and, with
 * hold_issuer != 0, makes the MMA-issuing thread first wait for a device
 * flag that nothing sets, so that the bound runs out on purpose.           */
fmma_status fmma_debug_m2l_wait(fmma_ctx* ctx, long long wait_cycles,
                                int hold_issuer);

/* ---- timing -------------------------------------------------------------
 * Stage times of the last solve in ms (CUDA events on the context stream),
 * in the reference's stage names (src/fmm.cpp:60-141): index 0..8 =
 * tree, P2M, M2M, M2L, L2L, L2P, P2P, exact, total.                         */
#define FMMA_NUM_STAGES 9
fmma_status fmma_stage_times(fmma_ctx* ctx, double* ms, int n);
const char* fmma_stage_name(int i);
/* Number of device kernels this library launched in the last solve.        */
int64_t fmma_last_launch_count(fmma_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for event timing by callers. */
void* fmma_ctx_stream(fmma_ctx* ctx);
/* M2L kernels of the last solve: summed CUDA-event time of the launches,
 * algorithmic flops (2 P^2 per target/source box pair and rhs), launches. */
fmma_status fmma_m2l_stats(fmma_ctx* ctx, double* kernel_ms, double* flops,
                           int64_t* launches);
/* Tree of the last fmm solve: M2L pairs over all levels, P2P point pairs,
 * non-empty leaves.                                                         */
fmma_status fmma_tree_stats(fmma_ctx* ctx, int64_t* m2l_pairs,
                            int64_t* p2p_pairs, int64_t* nleaf);
/* Per virtual level v (v = 0: leaves) of the last fmm solve's tree: boxes
 * holding points (`nbox[v]`) and M2L/L2L rows, the boxes holding targets
 * (`nrow[v]`); up to `cap` levels written, `*nlev` = levels in the tree.
 * Feeds the per-stage byte counts of the measurement; no counterpart in the
 * reference (its dense grid has 2^(d*l) boxes per level).                   */
fmma_status fmma_tree_levels(fmma_ctx* ctx, int cap, int* nlev, int64_t* nbox,
                             int64_t* nrow);

/* ---- user device functors ------------------------------------------------
 * The kernel-dependent stages (M2L operator tables, per-pair M2L, P2P, exact)
 * can be launched by a hook compiled in the caller's nvcc translation unit
 * (include/fmma/device.cuh instantiates them for a user __device__ functor);
 * replaces FMMA::set_fn with an arbitrary functor (include/fmma/fmma.hpp:65-87).
 * The hook launches on args->stream and returns a cudaError_t value.        */
enum {
  FMMA_USER_TABLE = 0,         /* tab[f][kl][km] = f(len*x_kl/2, len*(o_f + x_km/2)) */
  FMMA_USER_P2P = 1,           /* near field of every leaf row, FP64             */
  FMMA_USER_EXACT = 2,         /* direct sum                                       */
  FMMA_USER_M2L_PAIRWISE = 3,  /* M2L on absolute node coordinates (src/fmm_core.cpp:456-492) */
  FMMA_USER_NRNMM_FAR = 4      /* nrnmm far field (src/nrnmm.cpp:86-97)                  */
};

typedef struct fmma_user_launch {
  int what, dim, nrhs;
  void* stream;
  /* FMMA_USER_TABLE */
  double len;
  const double* node_all;      /* [P][dim] Chebyshev tensor nodes             */
  int P, npad, kpad, noff;
  const int* offv;             /* [noff][3] offsets (source box - target box)  */
  double* tab;                 /* [noff][npad][kpad], zero padding             */
  /* FMMA_USER_P2P: out[r][perm_t[t]] = pot[r][t] + sum_{near j} ws[r][j] f(x_t, y_j) */
  int64_t nrow;
  const int* row_box;
  const int* near;             /* [nrow][nnear] leaf box or -1                 */
  int nnear;
  const int *tb, *te, *sb, *se; /* leaf target / source ranges (sorted order)  */
  const double* tx;            /* [dim][nt] sorted targets                     */
  int64_t nt;
  const double* sx;            /* [dim][ns] sorted sources                     */
  int64_t ns;
  const double* ws;            /* [nrhs][ns] sorted weights                    */
  const double* pot;           /* [nrhs][nt] far field or NULL                 */
  const int* perm_t;
  void* out;                   /* [nrhs][nt] in the caller's type              */
  int out_f32;
  /* FMMA_USER_EXACT: out[r][i] = sum_j w[r][j] f(tgt[rows ? rows[i] : i], src[j]) */
  const void* tgt;             /* [nt][dim] caller type (out_f32)               */
  const void* src;             /* [ns][dim]                                     */
  const void* w;               /* [nrhs][ns] or NULL                            */
  const int64_t* rows;
  /* FMMA_USER_M2L_PAIRWISE: Wl[b] = sum_slots K(b, s) Wm[s] for the rows of a level */
  const int* il;               /* [nrow][nfar]                                  */
  int nfar, level;
  const uint64_t* key;         /* Morton keys of the level's boxes              */
  const double* origin;        /* cube origin [dim] (host pointer)              */
  double Len;
  const double* Wm;            /* [box][nrhs][kpad]                             */
  double* Wl;
  /* FMMA_USER_NRNMM_FAR: far[r][t] = sum over the boxes s with se[s] > sb[s]
   * that differ from box key[t] by more than one in some dimension of
   * sum_k Wm[s][r][k] f(x_t, y_sk), with x_t[q] = tx[q][t] (sorted targets),
   * y_sk[q] = gx[(q * grid_n + i_q(s)) * n + k_q]; boxes are numbered
   * row-major over grid_n^dim (dimension 0 most significant), node k has
   * digits k_q in base n (last dimension fastest).  Also uses dim, nrhs, P,
   * kpad, nt, tx, key, sb, se, Wm.                                           */
  int grid_n, n;
  const double* gx;            /* [dim][grid_n][n] node coordinates             */
  double* far;                 /* [nrhs][nt]                                    */
} fmma_user_launch;

typedef int (*fmma_user_hook)(const fmma_user_launch* args, void* user);

/* Installs a user kernel (hook != NULL) or returns to the built-in one
 * (hook == NULL).  `translation_invariant` says f(x,y) = g(x-y): the M2L
 * tables are then valid for any trans_sym flag.  Each call invalidates the
 * context's cached tables of earlier user kernels.                          */
fmma_status fmma_set_user_kernel(fmma_ctx* ctx, fmma_user_hook hook, void* user,
                                 int translation_invariant);

/* Kernel f given as a C++ expression (double) in x[q], y[q] (q < dim),
 * dx[q] = x[q] - y[q], r2 = |x - y|^2 and r = |x - y|, with the math
 * functions of CUDA device code (sqrt, exp, log, pow, ...), e.g.
 * "r2 > 0 ? 1 / r : 0" or "exp(-r2 / 0.01)".  The kernel-dependent stages
 * are compiled at run time (NVRTC, sm_100a) once per dimension, the 3-D
 * stages when this is called (a compile error is FMMA_ERR_INVALID_ARG with
 * the compiler's log in fmma_last_error), the others at their first solve.
 * `translation_invariant` declares f(x, y) = g(x - y) (table-mode M2L).
 * Replaces FMMA::set_fn with a callable (include/fmma/fmma.hpp:65-87) and
 * pyfmma's set_fn1/set_fn2 with a Python callable (cpython/pyfmma.cpp:150-151)
 * for kernels that can be written as a formula.                             */
fmma_status fmma_set_kernel_expr(fmma_ctx* ctx, const char* expr, int translation_invariant);

/* ---- global Chebyshev approximation -------------------------------------
 * Replaces fmma::CHEBYSHEV_APPROX<T,DIM> (include/fmma/chebyshev_approx.hpp,
 * src/chebyshev_approx.cpp:36-97): f on [-1,1]^dim ~ sum_i coef[i]
 * prod_q T_{i_q}(x_q), i_q in [0, nth], flat index i = sum_q i_q (nth+1)^q
 * (dimension 0 fastest, the reference's order for nodes and coefficients).
 *
 * fmma_cheb_nodes: the 1-D nodes x_k = cos((2k+1) pi / (2 nth + 2)),
 * k = 0..nth (host, no context); the fit point of flat index i has
 * coordinate q = x_{i_q}.
 * fmma_cheb_fit_d: coef[f][i] from values[f][i] = f(node i) for nfunc
 * functions: the exact solution of the reference's collocation system (the
 * reference iterates GCR to a squared residual of 1e-6).  values and coef
 * must not alias.
 * fmma_cheb_eval_d: out[f][p] = sum_i coef[f][i] prod_q T_{i_q}(pts[p][q])
 * (reference predict); a point outside [-1,1] is FMMA_ERR_INVALID_ARG (the
 * reference exits, src/math.cpp:14-26).  Limits: dim 1..3, nth <= 4095,
 * (nth+1)^dim <= 2^24.                                                      */
fmma_status fmma_cheb_nodes(int nth, double* nodes);
fmma_status fmma_cheb_fit_d(fmma_ctx* ctx, int dim, int nth, int nfunc,
                            const double* values, double* coef, int mem_kind);
fmma_status fmma_cheb_eval_d(fmma_ctx* ctx, int dim, int nth, int nfunc,
                             const double* coef, int64_t npts, const double* pts,
                             double* out, int mem_kind);

/* ------------------------------------------------------------------------
 * Allocation-free exact sum.  No counterpart in the reference: its exact
 * solver (src/fmma.cpp:80-94) is a host loop that resizes the caller's
 * result vector on every call.
 *
 * ans[r * n_tgt + i] = sum_j w[r * n_src + j] f(tgt_i, src_j) with a
 * built-in kernel, on the current device, enqueued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream).  All pointers are device
 * memory in fmma_solve_d's layout (tgt n_tgt x dim, w nrhs x n_src, w NULL =
 * unit weights).  The source range is split over blocks so that small target
 * sets fill the GPU; the partial sums live in a 16 MiB static device array,
 * so the call makes no device or host allocation.
 *
 * Limit: n_tgt * nrhs <= 262144 (FMMA_ERR_INVALID_ARG beyond, with the limit
 * in the message); larger target sets go through fmma_solve_d.
 * The first call on a device does its set-up (loading this entry point's
 * kernels, reading the SM count) and should come before any stream capture;
 * every call looks up the array's address in the current context, so calls
 * after a cudaDeviceReset find it again.
 * Calls whose executions overlap on one device (two streams, or two host
 * threads) share the array and race: order them on one stream or by events.
 * For callers that cannot allocate: code running while another component
 * owns the device memory budget (a caching allocator that has reserved it),
 * and loops that must not take cudaMalloc/cudaFree's implicit device-wide
 * synchronisation.                                                          */
fmma_status fmma_exact_noalloc_d(int dim, int kernel_id, double p0,
                                 int64_t n_tgt, const double* tgt,
                                 int64_t n_src, const double* src, int nrhs,
                                 const double* w, double* ans, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FMMA_B200_H */
