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
// pair: -1 the context's option, 0 the 1-SM kernel, 1 the 2-SM kernel where the level allows it;
// units: (slot, K chunk) units per pipeline stage, -1 the context's option
void m2l_level_tc(fmma_ctx* ctx, bool bf16, int pair, int units, const Level& Lv, int v, int nfar, const int* slot_off,
                  int P,
                  int Kpad64, int R, const double* Wm64, double* Wl64, const double* tab64, int Npad64,
                  const std::string& tabkey, int noff, int ntab);

// Mixed-precision near field: FP32 box-local evaluations, compensated sums.
// wst_ready: the FP32 weight rows were written by gather_weights_mixed.
template <typename T>
void p2p_mixed(fmma_ctx* ctx, int d, const double* tx, const double* sx, const double* ws, int R, const double* pot,
               T* out, bool wst_ready = false);

// ws[r][j] = w[r][perm[j]] plus the mixed near field's FP32 weight rows, one pass.
template <typename T>
void gather_weights_mixed(fmma_ctx* ctx, const T* w, const int* perm, int64_t ns, int R, double* ws);

template <typename T>
void solve_exact(fmma_ctx* ctx, int dim, int64_t nt, const T* tgt, int64_t ns, const T* src, int R, const T* w,
                 T* ans, const int64_t* rows);

// FP64 near field over tr's leaf near lists (built-in kernel or user hook):
// ans[r][perm_t[t]] = pot[r][t] + sum over near sources (pot may be NULL).
template <typename T>
void near_field_f64(fmma_ctx* ctx, int d, int R, const Tree& tr, const double* tx, const double* sx, const double* ws,
                    const double* pot, T* ans);

// out[q][i] = p[perm[i]][q] (FP64); out[r][i] = w[r][perm[i]] (1 when w is NULL).
template <typename T>
void launch_gather_points(fmma_ctx* ctx, const T* p, const int* perm, int64_t n, int d, double* out);
template <typename T>
void launch_gather_weights(fmma_ctx* ctx, const T* w, const int* perm, int64_t ns, int R, double* out);

// The nrnmm solver on one grid of nrn^dim boxes (src/nrnmm.cpp:13-102).
template <typename T>
void solve_nrnmm(fmma_ctx* ctx, const SolveArgs& a, int nrn, int64_t nt, const T* tgt, int64_t ns, const T* src,
                 const T* w, T* ans);
// Default boxes per dimension: (int)(sqrt(3) * ns^(1/(2 dim))) + 1, with ns
// rounded to the caller's type first (src/nrnmm.cpp:21-23).
int nrnmm_default_grid(int64_t ns, int dim, bool isf);

double* cached_op(fmma_ctx* ctx, const std::string& key, size_t bytes, bool* fresh);
std::string op_key(const char* kind, fmma_ctx* ctx, int d, int n, double len, int a, int b);
std::vector<int4> m2l_tiles(const Level& Lv, int R, int TM);

}  // namespace fmma_b200
