// solver.cuh — solver entry points shared between the C ABI and the stages.
#pragma once

#include <string>
#include <vector>

#include "fmma_internal.cuh"

namespace fmma_b200 {

template <typename T>
void solve_fmm(fmma_ctx* ctx, const SolveArgs& a, int64_t nt, const T* tgt, int64_t ns, const T* src, const T* w,
               T* ans);

template <typename T>
void solve_fmm_mixed(fmma_ctx* ctx, const SolveArgs& a, int64_t nt, const T* tgt, int64_t ns, const T* src,
                     const T* w, T* ans);

template <typename T>
void solve_exact(fmma_ctx* ctx, int dim, int64_t nt, const T* tgt, int64_t ns, const T* src, int R, const T* w,
                 T* ans, const int64_t* rows);

double* cached_op(fmma_ctx* ctx, const std::string& key, size_t bytes, bool* fresh);
std::string op_key(const char* kind, fmma_ctx* ctx, int d, int n, double len, int a, int b);
std::vector<int4> m2l_tiles(const Level& Lv, int nclass, int R, int TM);

}  // namespace fmma_b200
