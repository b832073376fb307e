// capi.cu — the C ABI of include/fmma_b200.h.
//
// Validation follows the reference's contract (src/fmm.cpp:20-35,
// src/fmma.cpp:143-186) but reports errors as status codes instead of
// exit(EXIT_FAILURE).
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "fmma_internal.cuh"
#include "kernels.cuh"
#include "solver.cuh"

using namespace fmma_b200;

namespace fmma_b200 {
static thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }
}  // namespace fmma_b200

namespace {

template <typename F>
fmma_status guarded(F&& f) {
  try {
    f();
    return FMMA_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return FMMA_ERR_OOM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FMMA_ERR_CUDA;
  }
}

void use_device(fmma_ctx* ctx) {
  FMMA_REQUIRE(ctx != nullptr, "null context");
  FMMA_CHECK_CUDA(cudaSetDevice(ctx->device));
}

// Copies a caller buffer to device scratch when it lives in host memory.
template <typename T>
const T* to_device(fmma_ctx* ctx, const char* name, const T* p, size_t count, int mem_kind) {
  if (mem_kind == FMMA_MEM_DEVICE || p == nullptr || count == 0) return p;
  T* d = ctx_buf_t<T>(ctx, name, count);
  FMMA_CHECK_CUDA(cudaMemcpyAsync(d, p, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream));
  return d;
}

// Morton codes occupy the low 52 bits of a key, box coordinates are ints.
int max_depth_for(int dim) { return dim == 3 ? 18 : (dim == 2 ? 27 : 31); }

void check_common(fmma_ctx* ctx, int dim, int64_t nt, const void* tgt, int64_t ns, const void* src, int mem_kind) {
  FMMA_REQUIRE(ctx != nullptr, "null context");
  FMMA_REQUIRE(dim >= 1 && dim <= 3, "dim must be 1, 2 or 3");
  FMMA_REQUIRE(nt >= 0 && ns >= 0, "negative point count");
  FMMA_REQUIRE(nt + ns < ((int64_t)1 << 31), "n_tgt + n_src must be below 2^31");
  FMMA_REQUIRE(nt == 0 || tgt != nullptr, "null target pointer");
  FMMA_REQUIRE(ns == 0 || src != nullptr, "null source pointer");
  FMMA_REQUIRE(mem_kind == FMMA_MEM_HOST || mem_kind == FMMA_MEM_DEVICE, "bad mem_kind");
  FMMA_REQUIRE(!(ctx->kernel_id == FMMA_KERNEL_INV_DIFF && dim != 1), "kernel 1/(x-y) is one-dimensional");
}

template <typename T>
fmma_status solve_impl(fmma_ctx* ctx, int dim, int solver, int poly_ord, int depth, int trans_sym, int precision,
                       int64_t nt, const T* tgt, int64_t ns, const T* src, int nrhs, const T* w, T* ans,
                       int mem_kind, int* depth_used) {
  return guarded([&] {
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    if (solver != FMMA_SOLVER_EXACT && solver != FMMA_SOLVER_FMM && solver != FMMA_SOLVER_TREE &&
        solver != FMMA_SOLVER_NRNMM)
      throw Error(FMMA_ERR_UNSUPPORTED_SOLVER, "solver type " + std::to_string(solver) +
                                                   " is not available: exact, fmm, tree and nrnmm run on the GPU");
    FMMA_REQUIRE(nrhs >= 1 && nrhs <= 64, "nrhs must be in [1, 64]");
    FMMA_REQUIRE(nt == 0 || ans != nullptr, "null ans pointer");
    FMMA_REQUIRE(precision >= FMMA_PREC_FP64 && precision <= FMMA_PREC_MIXED_BF16X3, "bad precision");
    if (solver == FMMA_SOLVER_TREE) {
      FMMA_REQUIRE(ctx->kernel_id != kUserKernel, "the tree solver runs built-in kernels");
      precision = FMMA_PREC_FP64;  // M2P and P2P in FP64
    }
    if (solver == FMMA_SOLVER_NRNMM) precision = FMMA_PREC_FP64;
    const int n = poly_ord + 1;
    int P = 1;
    for (int q = 0; q < dim; ++q) P *= n;
    if (solver == FMMA_SOLVER_FMM || solver == FMMA_SOLVER_TREE) {
      FMMA_REQUIRE(poly_ord >= 0 && n <= kMaxNodes, "poly_ord must be in [0, 15]");
      FMMA_REQUIRE(P <= 512, "at most 512 Chebyshev nodes per box (poly_ord <= 7 in 3D)");
      if (depth <= 0) depth = nt > 0 ? fmma_default_depth(nt, dim) : 1;
      FMMA_REQUIRE(depth <= max_depth_for(dim), "Depth too large for 64-bit Morton keys");
    }
    if (solver == FMMA_SOLVER_NRNMM) {
      // `depth` carries nrn_N, the boxes per dimension (src/nrnmm.cpp:20-22)
      FMMA_REQUIRE(poly_ord >= 0 && n <= kMaxNodes && n * dim <= 32, "poly_ord must be in [0, 15] (9 in 3D)");
      FMMA_REQUIRE(P <= 512, "at most 512 Chebyshev nodes per box (poly_ord <= 7 in 3D)");
      if (depth <= 0) depth = nrnmm_default_grid(ns, dim, sizeof(T) == 4);
      int64_t nbox = 1;
      for (int q = 0; q < dim; ++q) {
        nbox *= depth;
        FMMA_REQUIRE(nbox <= ((int64_t)1 << 28), "nrn_N^dim must be at most 2^28 boxes");
      }
    }
    if (depth_used) *depth_used = depth;
    use_device(ctx);
    stages_reset(ctx);
    stage_begin(ctx, ST_TOTAL);
    const size_t cnt_w = (size_t)nrhs * (size_t)ns;
    const T* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const T* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    const T* dw = to_device(ctx, "in_w", w, cnt_w, mem_kind);
    T* da = mem_kind == FMMA_MEM_DEVICE ? ans : ctx_buf_t<T>(ctx, "out_ans", (size_t)(nt * nrhs) + 1);
    if (nt > 0) {
      if (ns == 0) {
        FMMA_CHECK_CUDA(cudaMemsetAsync(da, 0, sizeof(T) * (size_t)(nt * nrhs), ctx->stream));
      } else if (solver == FMMA_SOLVER_NRNMM) {
        SolveArgs a{dim, n, P, depth, trans_sym, precision, nrhs, ctx->kernel_id, ctx->p0};
        solve_nrnmm<T>(ctx, a, depth, nt, dt, ns, ds, dw, da);
      } else if (solver == FMMA_SOLVER_EXACT) {
        stage_begin(ctx, ST_EXACT);
        solve_exact<T>(ctx, dim, nt, dt, ns, ds, nrhs, dw, da, nullptr);
        stage_end(ctx, ST_EXACT);
      } else {
        SolveArgs a{dim, n, P, depth, trans_sym, precision, nrhs, ctx->kernel_id, ctx->p0};
        a.tree = solver == FMMA_SOLVER_TREE ? 1 : 0;
        solve_fmm<T>(ctx, a, nt, dt, ns, ds, dw, da);
      }
      if (mem_kind == FMMA_MEM_HOST)
        FMMA_CHECK_CUDA(cudaMemcpyAsync(ans, da, sizeof(T) * (size_t)(nt * nrhs), cudaMemcpyDeviceToHost, ctx->stream));
    }
    stage_end(ctx, ST_TOTAL);
    stages_collect(ctx);
  });
}

}  // namespace

extern "C" {

const char* fmma_last_error(void) { return g_last_error.c_str(); }

const char* fmma_version(void) { return "fmma_b200 0.1.0 (sm_100a)"; }

int fmma_default_depth(int64_t n_tgt, int dim) {
  if (n_tgt <= 0 || dim <= 0) return 1;
  int D = (int)(std::log((double)n_tgt) / dim) + 1;
  return D <= 0 ? 1 : D;
}

fmma_status fmma_ctx_create(int device, fmma_ctx** out) {
  return guarded([&] {
    FMMA_REQUIRE(out != nullptr, "null output pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Error(FMMA_ERR_NO_DEVICE, "no CUDA device available");
    }
    FMMA_REQUIRE(device >= 0 && device < count, "device index out of range");
    FMMA_CHECK_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FMMA_CHECK_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
      throw Error(FMMA_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100 (B200) class");
    fmma_ctx* c = new fmma_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    FMMA_CHECK_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2 * FMMA_NUM_STAGES; ++i) FMMA_CHECK_CUDA(cudaEventCreate(&c->ev[i]));
    *out = c;
  });
}

fmma_status fmma_ctx_destroy(fmma_ctx* ctx) {
  if (!ctx) return FMMA_OK;
  return guarded([&] {
    cudaSetDevice(ctx->device);
    release_device_memory(ctx);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->up_host) cudaFreeHost(ctx->up_host);
    for (int i = 0; i < 2 * FMMA_NUM_STAGES; ++i)
      if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (int i = 0; i < 2 * fmma_ctx::kMaxTimed; ++i)
      if (ctx->kev[i]) cudaEventDestroy(ctx->kev[i]);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
  });
}

fmma_status fmma_set_allocator(fmma_ctx* ctx, fmma_alloc_fn alloc, fmma_free_fn free_fn, void* user) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    FMMA_REQUIRE(alloc == nullptr || free_fn != nullptr, "an allocator needs a free function");
    use_device(ctx);
    release_device_memory(ctx);  // through the allocator that made them
    ctx->tree = Tree{};          // its arrays lived in the released scratch
    ctx->alloc_fn = alloc;
    ctx->free_fn = alloc ? free_fn : nullptr;
    ctx->alloc_user = alloc ? user : nullptr;
  });
}

fmma_status fmma_set_m2l_options(fmma_ctx* ctx, int pair, int stages, int group, int units) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    FMMA_REQUIRE(pair >= -1 && pair <= 1, "pair must be -1, 0 or 1");
    FMMA_REQUIRE(stages == 0 || (stages >= 2 && stages <= 8), "stages must be 0 or 2..8");
    FMMA_REQUIRE(group >= 0 && group <= 189, "group must be 0..189");
    FMMA_REQUIRE(units >= 0 && units <= 4, "units must be 0..4");
    ctx->tc_pair = pair;
    ctx->tc_stages = stages;
    ctx->tc_group = group;
    ctx->tc_units = units;
  });
}

fmma_status fmma_set_schedule_options(fmma_ctx* ctx, int m2l_split, int l2p_mode) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    FMMA_REQUIRE(m2l_split >= 0 && m2l_split <= 3, "m2l_split must be 0..3");
    FMMA_REQUIRE(l2p_mode >= 0 && l2p_mode <= 2, "l2p_mode must be 0..2");
    ctx->tc_split = m2l_split;
    ctx->l2p_mode = l2p_mode;
  });
}

fmma_status fmma_debug_m2l_wait(fmma_ctx* ctx, long long wait_cycles, int hold_issuer) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    ctx->tc_wait_cycles = wait_cycles > 0 ? wait_cycles : 0;
    ctx->tc_hold = hold_issuer != 0;
  });
}

fmma_status fmma_set_kernel(fmma_ctx* ctx, int kernel_id, double p0) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    FMMA_REQUIRE(kernel_id >= 0 && kernel_id < FMMA_KERNEL_COUNT, "unknown kernel id");
    ctx->user_hook = nullptr;
    ctx->user_ptr = nullptr;
    ctx->user_own.reset();
    if (kernel_id == FMMA_KERNEL_GAUSSIAN) FMMA_REQUIRE(p0 > 0.0, "Gaussian width p0 must be > 0");
    if (kernel_id == FMMA_KERNEL_MULTIQUADRIC) FMMA_REQUIRE(p0 >= 0.0, "multiquadric shift p0 must be >= 0");
    ctx->kernel_id = kernel_id;
    ctx->p0 = p0;
  });
}

fmma_status fmma_set_user_kernel(fmma_ctx* ctx, fmma_user_hook hook, void* user, int translation_invariant) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    ctx->user_own.reset();
    if (hook == nullptr) {
      if (ctx->kernel_id == kUserKernel) ctx->kernel_id = FMMA_KERNEL_INV_R;
      ctx->user_hook = nullptr;
      ctx->user_ptr = nullptr;
      return;
    }
    ctx->user_hook = hook;
    ctx->user_ptr = user;
    ctx->user_ti = translation_invariant ? 1 : 0;
    ctx->user_gen++;
    ctx->kernel_id = kUserKernel;
    ctx->p0 = 0.0;
  });
}

fmma_status fmma_solve_d(fmma_ctx* ctx, int dim, int solver, int poly_ord, int depth, int trans_sym, int precision,
                         int64_t n_tgt, const double* tgt, int64_t n_src, const double* src, int nrhs,
                         const double* w, double* ans, int mem_kind, int* depth_used) {
  return solve_impl<double>(ctx, dim, solver, poly_ord, depth, trans_sym, precision, n_tgt, tgt, n_src, src, nrhs, w,
                            ans, mem_kind, depth_used);
}

fmma_status fmma_solve_f(fmma_ctx* ctx, int dim, int solver, int poly_ord, int depth, int trans_sym, int precision,
                         int64_t n_tgt, const float* tgt, int64_t n_src, const float* src, int nrhs, const float* w,
                         float* ans, int mem_kind, int* depth_used) {
  return solve_impl<float>(ctx, dim, solver, poly_ord, depth, trans_sym, precision, n_tgt, tgt, n_src, src, nrhs, w,
                           ans, mem_kind, depth_used);
}

#define FMMA_SOLVE_DIM(NAME, T, DIM, BASE)                                                                       \
  fmma_status NAME(fmma_ctx* ctx, int solver, int poly_ord, int depth, int trans_sym, int precision, int64_t nt,  \
                   const T* tgt, int64_t ns, const T* src, int nrhs, const T* w, T* ans, int mem_kind,            \
                   int* depth_used) {                                                                            \
    return BASE(ctx, DIM, solver, poly_ord, depth, trans_sym, precision, nt, tgt, ns, src, nrhs, w, ans, mem_kind, \
                depth_used);                                                                                     \
  }
FMMA_SOLVE_DIM(fmma_solve_d1, double, 1, fmma_solve_d)
FMMA_SOLVE_DIM(fmma_solve_d2, double, 2, fmma_solve_d)
FMMA_SOLVE_DIM(fmma_solve_d3, double, 3, fmma_solve_d)
FMMA_SOLVE_DIM(fmma_solve_f1, float, 1, fmma_solve_f)
FMMA_SOLVE_DIM(fmma_solve_f2, float, 2, fmma_solve_f)
FMMA_SOLVE_DIM(fmma_solve_f3, float, 3, fmma_solve_f)
#undef FMMA_SOLVE_DIM

fmma_status fmma_solve_grad_d(fmma_ctx* ctx, int dim, int solver, int poly_ord, int depth, int trans_sym,
                              int precision, int64_t nt, const double* tgt, int64_t ns, const double* src, int nrhs,
                              const double* w, double* ans, double* grad, int mem_kind, int* depth_used) {
  return guarded([&] {
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    FMMA_REQUIRE(solver == FMMA_SOLVER_EXACT || solver == FMMA_SOLVER_FMM, "solver must be exact or fmm");
    FMMA_REQUIRE(nrhs >= 1 && nrhs <= 64, "nrhs must be in [1, 64]");
    FMMA_REQUIRE(nt == 0 || grad != nullptr, "null grad pointer");
    FMMA_REQUIRE(ctx->kernel_id != kUserKernel, "gradients need a built-in kernel");
    const int n = poly_ord + 1;
    int P = 1;
    for (int q = 0; q < dim; ++q) P *= n;
    if (solver == FMMA_SOLVER_FMM) {
      FMMA_REQUIRE(poly_ord >= 0 && n <= kMaxNodes && P <= 512, "bad poly_ord");
      if (depth <= 0) depth = nt > 0 ? fmma_default_depth(nt, dim) : 1;
      FMMA_REQUIRE(depth <= max_depth_for(dim), "Depth too large for 64-bit Morton keys");
    }
    if (depth_used) *depth_used = depth;
    use_device(ctx);
    stages_reset(ctx);
    stage_begin(ctx, ST_TOTAL);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    const double* dw = to_device(ctx, "in_w", w, (size_t)nrhs * (size_t)ns, mem_kind);
    double* da = ans == nullptr ? nullptr
                 : mem_kind == FMMA_MEM_DEVICE ? ans : ctx_buf_t<double>(ctx, "out_ans", (size_t)(nt * nrhs) + 1);
    double* dg = mem_kind == FMMA_MEM_DEVICE ? grad : ctx_buf_t<double>(ctx, "out_grad", (size_t)(nt * nrhs * dim) + 1);
    if (nt > 0) {
      if (ns == 0) {
        if (da) FMMA_CHECK_CUDA(cudaMemsetAsync(da, 0, sizeof(double) * (size_t)(nt * nrhs), ctx->stream));
        FMMA_CHECK_CUDA(cudaMemsetAsync(dg, 0, sizeof(double) * (size_t)(nt * nrhs * dim), ctx->stream));
      } else if (solver == FMMA_SOLVER_EXACT) {
        stage_begin(ctx, ST_EXACT);
        if (da) solve_exact<double>(ctx, dim, nt, dt, ns, ds, nrhs, dw, da, nullptr);
        solve_exact_grad(ctx, dim, nt, dt, ns, ds, nrhs, dw, dg, nullptr);
        stage_end(ctx, ST_EXACT);
      } else {
        SolveArgs a{dim, n, P, depth, trans_sym, precision, nrhs, ctx->kernel_id, ctx->p0};
        solve_fmm<double>(ctx, a, nt, dt, ns, ds, dw, da, dg);
      }
      if (mem_kind == FMMA_MEM_HOST) {
        if (da) FMMA_CHECK_CUDA(cudaMemcpyAsync(ans, da, sizeof(double) * (size_t)(nt * nrhs), cudaMemcpyDeviceToHost, ctx->stream));
        FMMA_CHECK_CUDA(cudaMemcpyAsync(grad, dg, sizeof(double) * (size_t)(nt * nrhs * dim), cudaMemcpyDeviceToHost, ctx->stream));
      }
    }
    stage_end(ctx, ST_TOTAL);
    stages_collect(ctx);
  });
}

// offsets: host arrays [nprob + 1]; the point arrays live in mem_kind memory
static void forest_offsets(int nprob, const int64_t* toff, const int64_t* soff, std::vector<int64_t>* vt,
                           std::vector<int64_t>* vs) {
  FMMA_REQUIRE(nprob >= 1 && nprob <= kMaxProblems, "nprob must be in [1, 4096]");
  FMMA_REQUIRE(toff && soff, "null offsets");
  vt->assign(toff, toff + nprob + 1);
  vs->assign(soff, soff + nprob + 1);
  FMMA_REQUIRE((*vt)[0] == 0 && (*vs)[0] == 0, "offsets start at 0");
  for (int p = 0; p < nprob; ++p)
    FMMA_REQUIRE((*vt)[(size_t)p + 1] >= (*vt)[(size_t)p] && (*vs)[(size_t)p + 1] >= (*vs)[(size_t)p],
                 "offsets must not decrease");
}

fmma_status fmma_forest_depths_d(fmma_ctx* ctx, int dim, int nprob, const int64_t* toff, const double* tgt,
                                 const int64_t* soff, const double* src, int leaf_cap, int mem_kind, int* depths) {
  return guarded([&] {
    std::vector<int64_t> vt, vs;
    forest_offsets(nprob, toff, soff, &vt, &vs);
    const int64_t nt = vt.back(), ns = vs.back();
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    FMMA_REQUIRE(leaf_cap >= 1 && depths, "bad arguments");
    use_device(ctx);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    std::vector<int> cur((size_t)nprob, 1), done((size_t)nprob, 0);
    int remaining = nprob;
    for (int L = 1; L <= max_depth_for(dim) && remaining > 0; ++L) {
      for (int p = 0; p < nprob; ++p)
        if (!done[(size_t)p]) cur[(size_t)p] = L;
      std::vector<int> mt, ms;
      leaf_occupancy<double>(ctx, dim, vt, dt, vs, ds, cur, &mt, &ms);
      for (int p = 0; p < nprob; ++p)
        if (!done[(size_t)p] && mt[(size_t)p] <= leaf_cap && ms[(size_t)p] <= leaf_cap) {
          done[(size_t)p] = 1;
          --remaining;
        }
    }
    FMMA_REQUIRE(remaining == 0, "leaf cap cannot be met within the depth limit");
    for (int p = 0; p < nprob; ++p) depths[p] = cur[(size_t)p];
  });
}

fmma_status fmma_forest_solve_d(fmma_ctx* ctx, int dim, int nprob, const int64_t* toff, const double* tgt,
                                const int64_t* soff, const double* src, int nrhs, const double* w, double* ans,
                                int poly_ord, const int* depths, int trans_sym, int precision, int mem_kind) {
  return guarded([&] {
    std::vector<int64_t> vt, vs;
    forest_offsets(nprob, toff, soff, &vt, &vs);
    const int64_t nt = vt.back(), ns = vs.back();
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    FMMA_REQUIRE(ctx->kernel_id != kUserKernel, "forests take built-in kernels");
    FMMA_REQUIRE(nrhs >= 1 && nrhs <= 64, "nrhs must be in [1, 64]");
    FMMA_REQUIRE(nt == 0 || ans != nullptr, "null ans pointer");
    FMMA_REQUIRE(depths != nullptr, "null depths");
    FMMA_REQUIRE(precision >= FMMA_PREC_FP64 && precision <= FMMA_PREC_MIXED_BF16X3, "bad precision");
    const int n = poly_ord + 1;
    int P = 1;
    for (int q = 0; q < dim; ++q) P *= n;
    FMMA_REQUIRE(poly_ord >= 0 && n <= kMaxNodes && P <= 512, "bad poly_ord");
    std::vector<int> dep(depths, depths + nprob);
    for (int p = 0; p < nprob; ++p) FMMA_REQUIRE(dep[(size_t)p] >= 1 && dep[(size_t)p] <= max_depth_for(dim), "bad depth");
    use_device(ctx);
    stages_reset(ctx);
    stage_begin(ctx, ST_TOTAL);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    const double* dw = to_device(ctx, "in_w", w, (size_t)nrhs * (size_t)ns, mem_kind);
    double* da = mem_kind == FMMA_MEM_DEVICE ? ans : ctx_buf_t<double>(ctx, "out_ans", (size_t)(nt * nrhs) + 1);
    if (nt > 0) {
      if (ns == 0) {
        FMMA_CHECK_CUDA(cudaMemsetAsync(da, 0, sizeof(double) * (size_t)(nt * nrhs), ctx->stream));
      } else {
        SolveArgs a{dim, n, P, 0, trans_sym, precision, nrhs, ctx->kernel_id, ctx->p0};
        solve_forest<double>(ctx, a, vt, dt, vs, ds, dep, dw, da, nullptr, true);
      }
      if (mem_kind == FMMA_MEM_HOST)
        FMMA_CHECK_CUDA(cudaMemcpyAsync(ans, da, sizeof(double) * (size_t)(nt * nrhs), cudaMemcpyDeviceToHost, ctx->stream));
    }
    stage_end(ctx, ST_TOTAL);
    stages_collect(ctx);
  });
}

fmma_status fmma_exact_rows_d(fmma_ctx* ctx, int dim, int64_t nrows, const int64_t* rows, int64_t n_tgt,
                              const double* tgt, int64_t n_src, const double* src, int nrhs, const double* w,
                              double* ans, int mem_kind) {
  return guarded([&] {
    check_common(ctx, dim, n_tgt, tgt, n_src, src, mem_kind);
    FMMA_REQUIRE(nrows >= 0 && (nrows == 0 || rows != nullptr), "bad rows");
    FMMA_REQUIRE(nrhs >= 1 && nrhs <= 64, "nrhs must be in [1, 64]");
    use_device(ctx);
    stages_reset(ctx);
    stage_begin(ctx, ST_TOTAL);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(n_tgt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(n_src * dim), mem_kind);
    const double* dw = to_device(ctx, "in_w", w, (size_t)nrhs * (size_t)n_src, mem_kind);
    const int64_t* dr = to_device(ctx, "in_rows", rows, (size_t)nrows, mem_kind);
    double* da = mem_kind == FMMA_MEM_DEVICE ? ans : ctx_buf_t<double>(ctx, "out_rows", (size_t)(nrows * nrhs) + 1);
    if (nrows > 0) {
      stage_begin(ctx, ST_EXACT);
      if (n_src == 0)
        FMMA_CHECK_CUDA(cudaMemsetAsync(da, 0, sizeof(double) * (size_t)(nrows * nrhs), ctx->stream));
      else
        solve_exact<double>(ctx, dim, nrows, dt, n_src, ds, nrhs, dw, da, dr);
      stage_end(ctx, ST_EXACT);
      if (mem_kind == FMMA_MEM_HOST)
        FMMA_CHECK_CUDA(cudaMemcpyAsync(ans, da, sizeof(double) * (size_t)(nrows * nrhs), cudaMemcpyDeviceToHost, ctx->stream));
    }
    stage_end(ctx, ST_TOTAL);
    stages_collect(ctx);
  });
}

fmma_status fmma_cheb_nodes(int nth, double* nodes) {
  return guarded([&] {
    FMMA_REQUIRE(nth >= 0 && nodes != nullptr, "need nth >= 0 and an output array");
    for (int k = 0; k <= nth; ++k) nodes[k] = std::cos((2.0 * k + 1.0) / (2 * nth + 2) * M_PI);
  });
}

static int64_t cheb_size(int dim, int nth) {
  FMMA_REQUIRE(dim >= 1 && dim <= 3, "dim must be 1, 2 or 3");
  FMMA_REQUIRE(nth >= 0 && nth <= 4095, "nth must be in [0, 4095]");
  int64_t size = 1;
  for (int q = 0; q < dim; ++q) {
    size *= nth + 1;
    FMMA_REQUIRE(size <= ((int64_t)1 << 24), "(nth + 1)^dim must be at most 2^24 coefficients");
  }
  return size;
}

fmma_status fmma_cheb_fit_d(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* values, double* coef,
                            int mem_kind) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    const int64_t size = cheb_size(dim, nth);
    FMMA_REQUIRE(nfunc >= 1 && (int64_t)nfunc * size <= ((int64_t)1 << 28), "nfunc * (nth + 1)^dim too large");
    FMMA_REQUIRE(values != nullptr && coef != nullptr && values != coef, "need distinct values and coef arrays");
    FMMA_REQUIRE(mem_kind == FMMA_MEM_HOST || mem_kind == FMMA_MEM_DEVICE, "bad mem_kind");
    use_device(ctx);
    const size_t total = (size_t)(size * nfunc);
    const double* dv = to_device(ctx, "cheb_in_values", values, total, mem_kind);
    double* dc = mem_kind == FMMA_MEM_DEVICE ? coef : ctx_buf_t<double>(ctx, "cheb_out_coef", total);
    cheb_fit(ctx, dim, nth, nfunc, dv, dc);
    if (mem_kind == FMMA_MEM_HOST)
      FMMA_CHECK_CUDA(cudaMemcpyAsync(coef, dc, sizeof(double) * total, cudaMemcpyDeviceToHost, ctx->stream));
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

fmma_status fmma_cheb_eval_d(fmma_ctx* ctx, int dim, int nth, int nfunc, const double* coef, int64_t npts,
                             const double* pts, double* out, int mem_kind) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    const int64_t size = cheb_size(dim, nth);
    FMMA_REQUIRE(nfunc >= 1 && (int64_t)nfunc * size <= ((int64_t)1 << 28), "nfunc * (nth + 1)^dim too large");
    FMMA_REQUIRE(npts >= 0 && npts < ((int64_t)1 << 40), "bad point count");
    FMMA_REQUIRE(coef != nullptr && (npts == 0 || (pts != nullptr && out != nullptr)), "null pointer");
    FMMA_REQUIRE(mem_kind == FMMA_MEM_HOST || mem_kind == FMMA_MEM_DEVICE, "bad mem_kind");
    if (npts == 0) return;
    use_device(ctx);
    const double* dc = to_device(ctx, "cheb_in_coef", coef, (size_t)(size * nfunc), mem_kind);
    const double* dp = to_device(ctx, "cheb_in_pts", pts, (size_t)(npts * dim), mem_kind);
    double* dout = mem_kind == FMMA_MEM_DEVICE ? out : ctx_buf_t<double>(ctx, "cheb_out", (size_t)(npts * nfunc));
    cheb_eval(ctx, dim, nth, nfunc, dc, npts, dp, dout);
    if (mem_kind == FMMA_MEM_HOST)
      FMMA_CHECK_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * (size_t)(npts * nfunc), cudaMemcpyDeviceToHost,
                                      ctx->stream));
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

fmma_status fmma_tree_export_d(fmma_ctx* ctx, int dim, int depth, int64_t nt, const double* tgt, int64_t ns,
                               const double* src, int64_t* tgt_box, int64_t* src_box, double* origin_len,
                               int mem_kind) {
  return guarded([&] {
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    FMMA_REQUIRE(depth >= 1 && depth <= max_depth_for(dim), "bad depth");
    FMMA_REQUIRE(nt + ns > 0, "no points");
    use_device(ctx);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    int64_t* tb = mem_kind == FMMA_MEM_DEVICE ? tgt_box : ctx_buf_t<int64_t>(ctx, "exp_tb", (size_t)nt + 1);
    int64_t* sb = mem_kind == FMMA_MEM_DEVICE ? src_box : ctx_buf_t<int64_t>(ctx, "exp_sb", (size_t)ns + 1);
    Cube c;
    export_bins<double>(ctx, dim, depth, nt, dt, ns, ds, tb, sb, &c);
    if (mem_kind == FMMA_MEM_HOST) {
      if (nt) FMMA_CHECK_CUDA(cudaMemcpyAsync(tgt_box, tb, sizeof(int64_t) * (size_t)nt, cudaMemcpyDeviceToHost, ctx->stream));
      if (ns) FMMA_CHECK_CUDA(cudaMemcpyAsync(src_box, sb, sizeof(int64_t) * (size_t)ns, cudaMemcpyDeviceToHost, ctx->stream));
    }
    FMMA_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (origin_len) {
      for (int q = 0; q < dim; ++q) origin_len[q] = c.origin[q];
      origin_len[dim] = c.Len;
    }
  });
}

// list queries on the tree of the last fmm solve
static void find_row(fmma_ctx* ctx, int level, int64_t box, bool near, int* row_out, int* nlist,
                     std::vector<int>& list, std::vector<uint64_t>& keys) {
  Tree& tr = ctx->tree;
  FMMA_REQUIRE(tr.valid && !tr.lev.empty() && tr.near != nullptr, "no fmm tree: run an fmm solve first");
  FMMA_REQUIRE(tr.nprob == 1, "list queries need a single-problem tree");
  FMMA_REQUIRE(level >= 2 && level < tr.depth0(), "level out of range");
  const int d = tr.dim;
  const Level& Lv = tr.real(level);
  const int64_t N = (int64_t)1 << level;
  int c[kMaxDim] = {0, 0, 0};
  int64_t bc = box;
  for (int q = d - 1; q >= 0; --q) { c[q] = (int)(bc % N); bc /= N; }
  FMMA_REQUIRE(box >= 0 && bc == 0, "box index out of range");
  uint64_t k = morton_encode(c, d, level);
  keys.resize((size_t)Lv.nbox);
  FMMA_CHECK_CUDA(cudaMemcpy(keys.data(), Lv.key, sizeof(uint64_t) * (size_t)Lv.nbox, cudaMemcpyDeviceToHost));
  auto it = std::lower_bound(keys.begin(), keys.end(), k);
  FMMA_REQUIRE(it != keys.end() && *it == k, "box holds no points");
  int b = (int)(it - keys.begin());
  int64_t nrow = near ? tr.nnear_rows : Lv.nrow;
  std::vector<int> rb((size_t)nrow);
  FMMA_CHECK_CUDA(cudaMemcpy(rb.data(), near ? tr.near_row_box : Lv.row_box, sizeof(int) * (size_t)nrow,
                             cudaMemcpyDeviceToHost));
  int row = -1;
  for (int64_t r = 0; r < nrow; ++r)
    if (rb[(size_t)r] == b) { row = (int)r; break; }
  FMMA_REQUIRE(row >= 0, "box holds no targets");
  int nl = near ? (d == 1 ? 3 : d == 2 ? 9 : 27) : far_tables(d).nfar;
  list.resize((size_t)nl);
  FMMA_CHECK_CUDA(cudaMemcpy(list.data(), (near ? tr.near : Lv.il) + (int64_t)row * nl, sizeof(int) * (size_t)nl,
                             cudaMemcpyDeviceToHost));
  *row_out = row;
  *nlist = nl;
}

static void emit_list(int d, int level, const std::vector<int>& list, const std::vector<uint64_t>& keys,
                      int64_t* out, int cap, int* count) {
  int cnt = 0;
  for (int s : list) {
    if (s < 0) continue;
    int c[kMaxDim] = {0, 0, 0};
    morton_decode(keys[(size_t)s], d, level, c);
    int64_t r = 0;
    for (int q = 0; q < d; ++q) r = (r << level) | c[q];
    if (cnt < cap) out[cnt] = r;
    ++cnt;
  }
  *count = cnt;
}

fmma_status fmma_interaction_list(fmma_ctx* ctx, int level, int64_t box, int64_t* out, int cap, int* count) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && out && count, "null argument");
    use_device(ctx);
    int row, nl;
    std::vector<int> list;
    std::vector<uint64_t> keys;
    find_row(ctx, level, box, false, &row, &nl, list, keys);
    emit_list(ctx->tree.dim, level, list, keys, out, cap, count);
  });
}

fmma_status fmma_near_list(fmma_ctx* ctx, int64_t box, int64_t* out, int cap, int* count) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && out && count, "null argument");
    use_device(ctx);
    int row, nl;
    std::vector<int> list;
    std::vector<uint64_t> keys;
    int level = ctx->tree.depth0() - 1;
    FMMA_REQUIRE(level >= 2, "near-list query needs Depth >= 3");
    find_row(ctx, level, box, true, &row, &nl, list, keys);
    emit_list(ctx->tree.dim, level, list, keys, out, cap, count);
  });
}

fmma_status fmma_max_leaf_occupancy_d(fmma_ctx* ctx, int dim, int depth, int64_t nt, const double* tgt, int64_t ns,
                                      const double* src, int mem_kind, int64_t* max_tgt, int64_t* max_src) {
  return guarded([&] {
    check_common(ctx, dim, nt, tgt, ns, src, mem_kind);
    FMMA_REQUIRE(depth >= 1 && depth <= max_depth_for(dim), "bad depth");
    FMMA_REQUIRE(nt + ns > 0, "no points");
    FMMA_REQUIRE(max_tgt && max_src, "null output");
    use_device(ctx);
    const double* dt = to_device(ctx, "in_tgt", tgt, (size_t)(nt * dim), mem_kind);
    const double* ds = to_device(ctx, "in_src", src, (size_t)(ns * dim), mem_kind);
    std::vector<int> mt, ms;
    leaf_occupancy<double>(ctx, dim, {0, nt}, dt, {0, ns}, ds, {depth}, &mt, &ms);
    *max_tgt = mt[0];
    *max_src = ms[0];
  });
}

fmma_status fmma_stage_times(fmma_ctx* ctx, double* ms, int n) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && ms, "null argument");
    for (int i = 0; i < n && i < FMMA_NUM_STAGES; ++i) ms[i] = ctx->stage_ms[i];
  });
}

const char* fmma_stage_name(int i) {
  static const char* names[FMMA_NUM_STAGES] = {"tree", "P2M", "M2M", "M2L", "L2L", "L2P", "P2P", "exact", "total"};
  return (i >= 0 && i < FMMA_NUM_STAGES) ? names[i] : "";
}

int64_t fmma_last_launch_count(fmma_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* fmma_ctx_stream(fmma_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

fmma_status fmma_m2l_stats(fmma_ctx* ctx, double* kernel_ms, double* flops, int64_t* launches) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && kernel_ms && flops && launches, "null argument");
    *kernel_ms = ctx->m2l_kernel_ms;
    *flops = ctx->m2l_flops;
    *launches = ctx->m2l_launches;
  });
}

fmma_status fmma_tree_stats(fmma_ctx* ctx, int64_t* m2l_pairs, int64_t* p2p_pairs, int64_t* nleaf) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && m2l_pairs && p2p_pairs && nleaf, "null argument");
    const Tree& tr = ctx->tree;
    FMMA_REQUIRE(tr.valid && !tr.lev.empty(), "no tree: run an fmm solve first");
    tree_read_pairs(ctx);
    int64_t s = 0;
    for (const Level& L : tr.lev) s += L.il_pairs;
    *m2l_pairs = s;
    *p2p_pairs = tr.p2p_pairs;
    *nleaf = tr.lev[0].nbox;
  });
}

fmma_status fmma_set_kernel_expr(fmma_ctx* ctx, const char* expr, int translation_invariant) {
  return guarded([&] {
    FMMA_REQUIRE(ctx != nullptr, "null context");
    set_kernel_expr(ctx, expr, translation_invariant);
    ctx->p0 = 0.0;
  });
}

fmma_status fmma_tree_levels(fmma_ctx* ctx, int cap, int* nlev, int64_t* nbox, int64_t* nrow) {
  return guarded([&] {
    FMMA_REQUIRE(ctx && nlev, "null argument");
    const Tree& tr = ctx->tree;
    FMMA_REQUIRE(tr.valid && !tr.lev.empty(), "no tree: run an fmm solve first");
    *nlev = (int)tr.lev.size();
    for (int v = 0; v < (int)tr.lev.size() && v < cap; ++v) {
      if (nbox) nbox[v] = tr.lev[(size_t)v].nbox;
      if (nrow) nrow[v] = tr.lev[(size_t)v].nrow;
    }
  });
}

}  // extern "C"
