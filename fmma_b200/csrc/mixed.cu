// mixed.cu — mixed-precision FMM (FP32 compensated P2P, split-precision
// tensor-core M2L).
#include "fmma_internal.cuh"
#include "solver.cuh"

namespace fmma_b200 {

template <typename T>
void solve_fmm_mixed(fmma_ctx*, const SolveArgs&, int64_t, const T*, int64_t, const T*, const T*, T*) {
  throw Error(FMMA_ERR_INVALID_ARG, "mixed precision is not built yet");
}

template void solve_fmm_mixed<double>(fmma_ctx*, const SolveArgs&, int64_t, const double*, int64_t, const double*,
                                      const double*, double*);
template void solve_fmm_mixed<float>(fmma_ctx*, const SolveArgs&, int64_t, const float*, int64_t, const float*,
                                     const float*, float*);

}  // namespace fmma_b200
