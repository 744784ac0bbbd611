// Batched blocked Cholesky kernels (potrf / posv), double instantiations.
#include "launch.cuh"
namespace tsdx {
namespace host {
template <> int run_chol<double>(const SolveArgs<double>& a, cudaStream_t st) { return run_blk<double, true>(a, st); }
template <> int run_potrs<double>(const SolveArgs<double>& a, cudaStream_t st) { return run_trs<double, false>(a, st); }
}  // namespace host
}  // namespace tsdx
