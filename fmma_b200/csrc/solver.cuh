// solver.cuh — solver entry points shared between the C ABI and the stages.
#pragma once

#include <string>
#include <vector>

#include "fmma_internal.cuh"

namespace fmma_b200 {

// ans may be NULL when grad is given (T = double only); grad is [R][nt][d].
template <typename T>
void solve_fmm(fmma_ctx* ctx, const SolveArgs& a, int64_t nt, const T* tgt, int64_t ns, const T* src, const T* w,
               T* ans, double* grad = nullptr);

void solve_exact_grad(fmma_ctx* ctx, int dim, int64_t nt, const double* tgt, int64_t ns, const double* src, int R,
                      const double* w, double* grad, const int64_t* rows);

// Forest solve: problem p owns tgt[toff[p]..toff[p+1]) and src[soff[p]..soff[p+1]);
// weights [R][ns_total], results [R][nt_total].
// build = false reuses ctx->tree and the gathered points (a plan's sweep).
template <typename T>
void solve_forest(fmma_ctx* ctx, const SolveArgs& a, const std::vector<int64_t>& toff, const T* tgt,
                  const std::vector<int64_t>& soff, const T* src, const std::vector<int>& depth, const T* w, T* ans,
                  double* grad, bool build);

// Tensor-core M2L of one virtual level (split-precision operands, FP64 output);
// tab64 holds ntab FP64 tables of noff operators each.
void m2l_level_tc(fmma_ctx* ctx, bool bf16, const Level& Lv, int v, int nfar, const int* slot_off, int P,
                  int Kpad64, int R, const double* Wm64, double* Wl64, const double* tab64, int Npad64,
                  const std::string& tabkey, int noff, int ntab);

// Mixed-precision near field: FP32 box-local evaluations, compensated sums.
template <typename T>
void p2p_mixed(fmma_ctx* ctx, int d, const double* tx, const double* sx, const double* ws, int R, const double* pot,
               T* out);

template <typename T>
void solve_exact(fmma_ctx* ctx, int dim, int64_t nt, const T* tgt, int64_t ns, const T* src, int R, const T* w,
                 T* ans, const int64_t* rows);

double* cached_op(fmma_ctx* ctx, const std::string& key, size_t bytes, bool* fresh);
std::string op_key(const char* kind, fmma_ctx* ctx, int d, int n, double len, int a, int b);
std::vector<int4> m2l_tiles(const Level& Lv, int R, int TM);

}  // namespace fmma_b200
