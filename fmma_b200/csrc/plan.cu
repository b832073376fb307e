// plan.cu — reusable solves: the tree, operator tables and buffers of a
// (forest) geometry are built once; the sweep (P2M .. P2P) is captured into a
// CUDA graph and replayed for new weights.  An autotuner times sweeps during
// the plan's warm-up and picks, per level, the M2L engine (FP64 DMMA, or the
// 1-SM or 2-SM tensor-core kernel with 1, 2 or 4 units per pipeline stage)
// and the slot split of small levels, and for the leaves the L2P lane layout
// (over targets, or over coefficients with the leaf L2L fused in); choices
// are remembered in the context's tuner cache (optionally persisted to a
// file).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "fmma_internal.cuh"
#include "solver.cuh"

using namespace fmma_b200;

struct fmma_plan {
  fmma_ctx* ctx = nullptr;  // private context: its tree and buffers belong to the plan
  SolveArgs a{};
  std::vector<int64_t> toff, soff;
  std::vector<int> depth;
  int64_t nt = 0, ns = 0;
  double* w_dev = nullptr;
  double* ans_dev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int*> err_flags;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double build_ms = 0.0, last_ms = 0.0;
  int levels_tc = 0, levels_f64 = 0;
};

namespace fmma_b200 {
void set_last_error(const std::string& m);
}

namespace {

template <typename F>
fmma_status guarded_plan(F&& f) {
  try {
    f();
    return FMMA_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FMMA_ERR_CUDA;
  }
}

std::string tuner_key(const SolveArgs& a, int v, const Level& Lv) {
  // rows rounded to a power of two: one decision per size class
  int64_t b = 1;
  while (b < Lv.nrow) b <<= 1;
  char buf[160];
  std::snprintf(buf, sizeof(buf), "m2l4_d%d_P%d_R%d_prec%d_rows%lld", a.dim, a.P, a.nrhs, a.precision, (long long)b);
  (void)v;
  return buf;
}

// Key of the leaf-evaluation choice: targets per leaf row rounded to a power
// of two, so problems of one shape class share the decision.
std::string tuner_key_l2p(const SolveArgs& a, int64_t nt, const Level& leaf) {
  int64_t b = 1;
  while (b * (leaf.nrow > 0 ? leaf.nrow : 1) < nt) b <<= 1;
  char buf[160];
  std::snprintf(buf, sizeof(buf), "l2p1_d%d_P%d_R%d_prec%d_tpr%lld", a.dim, a.P, a.nrhs, a.precision, (long long)b);
  return buf;
}

void tuner_load(fmma_ctx* ctx) {
  if (ctx->tuner_path.empty()) return;
  std::ifstream f(ctx->tuner_path);
  std::string k;
  int v;
  while (f >> k >> v) ctx->tuner[k] = v;
}

void tuner_save(fmma_ctx* ctx) {
  if (ctx->tuner_path.empty()) return;
  std::ofstream f(ctx->tuner_path);
  for (auto& kv : ctx->tuner) f << kv.first << " " << kv.second << "\n";
}

// One sweep without a tree build, returning the per-level M2L kernel times
// (and, in *leaf_ms, the L2L + L2P stage time: the fused leaf kernel moves
// the leaf L2L from one stage to the other).
std::vector<double> timed_sweep(fmma_plan* p, double* leaf_ms = nullptr) {
  fmma_ctx* c = p->ctx;
  stages_reset(c);
  solve_forest<double>(c, p->a, p->toff, nullptr, p->soff, nullptr, p->depth, p->w_dev, p->ans_dev, nullptr, false);
  stages_collect(c);
  if (leaf_ms) *leaf_ms = c->stage_ms[ST_L2L] + c->stage_ms[ST_L2P];
  std::vector<double> ms(c->tree.lev.size(), 0.0);
  for (int i = 0; i < c->ktimed; ++i)
    if (c->ktag[i] >= 0 && c->ktag[i] < (int)ms.size()) ms[(size_t)c->ktag[i]] += c->kms[i];
  return ms;
}

}  // namespace

extern "C" {

fmma_status fmma_plan_create_d(fmma_ctx* parent, int dim, int nprob, const int64_t* toff, const double* tgt,
                               const int64_t* soff, const double* src, int nrhs, int poly_ord, const int* depths,
                               int trans_sym, int precision, int autotune, int mem_kind, fmma_plan** out) {
  fmma_plan* p = nullptr;
  fmma_status st = guarded_plan([&] {
    FMMA_REQUIRE(parent && out && depths && toff && soff, "null argument");
    FMMA_REQUIRE(parent->kernel_id != kUserKernel, "plans take built-in kernels");
    FMMA_REQUIRE(nprob >= 1 && nprob <= kMaxProblems, "nprob must be in [1, 4096]");
    FMMA_REQUIRE(nrhs >= 1 && nrhs <= 64, "nrhs must be in [1, 64]");
    FMMA_REQUIRE(mem_kind == FMMA_MEM_HOST || mem_kind == FMMA_MEM_DEVICE, "bad mem_kind");
    FMMA_REQUIRE(precision >= FMMA_PREC_FP64 && precision <= FMMA_PREC_MIXED_BF16X3, "bad precision");
    *out = nullptr;
    p = new fmma_plan();
    FMMA_CHECK_CUDA(cudaSetDevice(parent->device));
    fmma_status cs = fmma_ctx_create(parent->device, &p->ctx);
    if (cs != FMMA_OK) throw Error(cs, fmma_last_error());
    fmma_ctx* c = p->ctx;
    c->kernel_id = parent->kernel_id;
    c->p0 = parent->p0;
    c->tuner = parent->tuner;
    c->tuner_path = parent->tuner_path;
    c->tc_pair = parent->tc_pair;
    c->tc_stages = parent->tc_stages;
    c->tc_group = parent->tc_group;
    c->tc_split = parent->tc_split;
    c->l2p_mode = parent->l2p_mode;
    c->tc_units = parent->tc_units;
    c->alloc_fn = parent->alloc_fn;
    c->free_fn = parent->free_fn;
    c->alloc_user = parent->alloc_user;
    p->toff.assign(toff, toff + nprob + 1);
    p->soff.assign(soff, soff + nprob + 1);
    p->depth.assign(depths, depths + nprob);
    p->nt = p->toff.back();
    p->ns = p->soff.back();
    FMMA_REQUIRE(p->nt > 0 && p->ns > 0, "a plan needs targets and sources");
    const int n = poly_ord + 1;
    int P = 1;
    for (int q = 0; q < dim; ++q) P *= n;
    FMMA_REQUIRE(dim >= 1 && dim <= 3 && poly_ord >= 0 && n <= kMaxNodes && P <= 512, "bad dim or poly_ord");
    p->a = SolveArgs{dim, n, P, 0, trans_sym, precision, nrhs, c->kernel_id, c->p0};
    FMMA_CHECK_CUDA(cudaEventCreate(&p->ev[0]));
    FMMA_CHECK_CUDA(cudaEventCreate(&p->ev[1]));

    // points into the plan's memory; zero weights for the warm-up
    double* dt = ctx_buf_t<double>(c, "plan_tgt", (size_t)(p->nt * dim));
    double* ds = ctx_buf_t<double>(c, "plan_src", (size_t)(p->ns * dim));
    const cudaMemcpyKind kind = mem_kind == FMMA_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    FMMA_CHECK_CUDA(cudaMemcpyAsync(dt, tgt, sizeof(double) * (size_t)(p->nt * dim), kind, c->stream));
    FMMA_CHECK_CUDA(cudaMemcpyAsync(ds, src, sizeof(double) * (size_t)(p->ns * dim), kind, c->stream));
    p->w_dev = ctx_buf_t<double>(c, "plan_w", (size_t)(p->ns * nrhs));
    p->ans_dev = ctx_buf_t<double>(c, "plan_ans", (size_t)(p->nt * nrhs));
    FMMA_CHECK_CUDA(cudaMemsetAsync(p->w_dev, 0, sizeof(double) * (size_t)(p->ns * nrhs), c->stream));

    // build + warm-up sweep (allocates every buffer, builds the tables)
    stages_reset(c);
    stage_begin(c, ST_TOTAL);
    solve_forest<double>(c, p->a, p->toff, dt, p->soff, ds, p->depth, p->w_dev, p->ans_dev, nullptr, true);
    stage_end(c, ST_TOTAL);
    stages_collect(c);
    p->build_ms = c->stage_ms[ST_TOTAL];

    // autotune (mixed precision only): per level the M2L engine and the slot
    // split of small levels, and the leaf evaluation
    const int V = (int)c->tree.lev.size();
    c->m2l_engine.assign((size_t)V, -1);
    c->m2l_split.assign((size_t)V, 0);  // 0: the context's split option
    if (precision != FMMA_PREC_FP64) {
      bool known = true;
      for (int v = 0; v < V; ++v) {
        const Level& Lv = c->tree.lev[(size_t)v];
        if (Lv.nrow == 0) continue;
        auto it = c->tuner.find(tuner_key(p->a, v, Lv));
        if (it == c->tuner.end()) known = false;
        else c->m2l_engine[(size_t)v] = it->second;
        auto is = c->tuner.find("split_" + tuner_key(p->a, v, Lv));
        if (is == c->tuner.end()) known = false;
        else c->m2l_split[(size_t)v] = is->second;
      }
      const std::string lkey = tuner_key_l2p(p->a, p->nt, c->tree.lev[0]);
      auto il = c->tuner.find(lkey);
      if (il == c->tuner.end()) known = false;
      else c->l2p_mode = il->second;
      if (autotune && !known) {
        // every level under each engine (FP64 DMMA; tensor-core 1-SM and
        // 2-SM with 1, 2 or 4 units per pipeline stage), a settling sweep
        // then a timed one; the fastest engine per level wins (the pipeline
        // depth and the drain group measured flat and stay at their
        // defaults: the group also moves the FP32 rounding)
        std::vector<double> t_eng[kM2LEngines];
        for (int e = 0; e < kM2LEngines; ++e) {
          std::fill(c->m2l_engine.begin(), c->m2l_engine.end(), e);
          timed_sweep(p);
          t_eng[e] = timed_sweep(p);
        }
        for (int v = 0; v < V; ++v) {
          const Level& Lv = c->tree.lev[(size_t)v];
          if (Lv.nrow == 0) continue;
          int choice = 0;
          for (int e = 1; e < kM2LEngines; ++e)
            if (t_eng[e][(size_t)v] < t_eng[choice][(size_t)v]) choice = e;
          c->m2l_engine[(size_t)v] = choice;
          c->tuner[tuner_key(p->a, v, Lv)] = choice;
        }
        // with the engines fixed: the slot split of the small 1-SM levels
        // (0 fill the SMs, 1 none, 2 half, 3 double; only levels with fewer
        // tiles than SMs run it, the others time alike) ...
        std::vector<double> t_split[4];
        for (int m = 0; m < 4; ++m) {
          std::fill(c->m2l_split.begin(), c->m2l_split.end(), m);
          timed_sweep(p);
          t_split[m] = timed_sweep(p);
        }
        for (int v = 0; v < V; ++v) {
          const Level& Lv = c->tree.lev[(size_t)v];
          if (Lv.nrow == 0) continue;
          int choice = 0;  // the default unless another is at least 3 % faster
          for (int m = 1; m < 4; ++m)
            if (t_split[m][(size_t)v] < 0.97 * t_split[choice][(size_t)v]) choice = m;
          c->m2l_split[(size_t)v] = choice;
          c->tuner["split_" + tuner_key(p->a, v, Lv)] = choice;
        }
        // ... and the leaf evaluation: lanes over targets or over coefficients
        double t_leaf[3] = {0.0, 0.0, 0.0};
        for (int m = 1; m <= 2; ++m) {
          c->l2p_mode = m;
          timed_sweep(p);
          timed_sweep(p, &t_leaf[m]);
        }
        c->l2p_mode = t_leaf[2] < t_leaf[1] ? 2 : 1;
        c->tuner[lkey] = c->l2p_mode;
        tuner_save(c);
        parent->tuner = c->tuner;
      }
      // one more uncaptured sweep with the final choices (allocations settle)
      timed_sweep(p);
    }
    for (int v = 0; v < V; ++v) {
      if (c->tree.lev[(size_t)v].nrow == 0) continue;
      if (precision != FMMA_PREC_FP64 && c->m2l_engine[(size_t)v] != 0) ++p->levels_tc;
      else ++p->levels_f64;
    }

    // capture the sweep
    FMMA_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    stages_reset(c);
    FMMA_CHECK_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->capturing = true;
    try {
      solve_forest<double>(c, p->a, p->toff, nullptr, p->soff, nullptr, p->depth, p->w_dev, p->ans_dev, nullptr,
                           false);
    } catch (...) {
      c->capturing = false;
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    c->capturing = false;
    FMMA_CHECK_CUDA(cudaStreamEndCapture(c->stream, &p->graph));
    FMMA_CHECK_CUDA(cudaGraphInstantiate(&p->exec, p->graph, 0));
    p->err_flags = c->m2l_err_flags;
    c->m2l_err_flags.clear();
    *out = p;
  });
  if (st != FMMA_OK && p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->ev[0]) cudaEventDestroy(p->ev[0]);
    if (p->ev[1]) cudaEventDestroy(p->ev[1]);
    if (p->ctx) fmma_ctx_destroy(p->ctx);
    delete p;
  }
  return st;
}

fmma_status fmma_plan_execute_d(fmma_plan* p, const double* w, double* ans, int mem_kind) {
  return guarded_plan([&] {
    FMMA_REQUIRE(p && p->exec && w && ans, "null argument");
    FMMA_REQUIRE(mem_kind == FMMA_MEM_HOST || mem_kind == FMMA_MEM_DEVICE, "bad mem_kind");
    fmma_ctx* c = p->ctx;
    FMMA_CHECK_CUDA(cudaSetDevice(c->device));
    const int R = p->a.nrhs;
    FMMA_CHECK_CUDA(cudaEventRecord(p->ev[0], c->stream));
    FMMA_CHECK_CUDA(cudaMemcpyAsync(p->w_dev, w, sizeof(double) * (size_t)(p->ns * R),
                                    mem_kind == FMMA_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                    c->stream));
    FMMA_CHECK_CUDA(cudaGraphLaunch(p->exec, c->stream));
    c->launches = 0;
    FMMA_CHECK_CUDA(cudaMemcpyAsync(ans, p->ans_dev, sizeof(double) * (size_t)(p->nt * R),
                                    mem_kind == FMMA_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                    c->stream));
    FMMA_CHECK_CUDA(cudaEventRecord(p->ev[1], c->stream));
    FMMA_CHECK_CUDA(cudaEventSynchronize(p->ev[1]));
    float ms = 0.f;
    FMMA_CHECK_CUDA(cudaEventElapsedTime(&ms, p->ev[0], p->ev[1]));
    p->last_ms = ms;
    check_m2l_errs(c, p->err_flags);
  });
}

fmma_status fmma_plan_stats(fmma_plan* p, double* build_ms, double* last_exec_ms, int* levels_tc, int* levels_f64,
                            int64_t* graph_nodes) {
  return guarded_plan([&] {
    FMMA_REQUIRE(p, "null plan");
    if (build_ms) *build_ms = p->build_ms;
    if (last_exec_ms) *last_exec_ms = p->last_ms;
    if (levels_tc) *levels_tc = p->levels_tc;
    if (levels_f64) *levels_f64 = p->levels_f64;
    if (graph_nodes) {
      size_t nn = 0;
      FMMA_CHECK_CUDA(cudaGraphGetNodes(p->graph, nullptr, &nn));
      *graph_nodes = (int64_t)nn;
    }
  });
}

fmma_status fmma_plan_destroy(fmma_plan* p) {
  if (!p) return FMMA_OK;
  return guarded_plan([&] {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->ev[0]) cudaEventDestroy(p->ev[0]);
    if (p->ev[1]) cudaEventDestroy(p->ev[1]);
    if (p->ctx) fmma_ctx_destroy(p->ctx);
    delete p;
  });
}

fmma_status fmma_set_tuner_cache(fmma_ctx* ctx, const char* path) {
  return guarded_plan([&] {
    FMMA_REQUIRE(ctx, "null context");
    ctx->tuner_path = path ? path : "";
    tuner_load(ctx);
  });
}

}  // extern "C"
