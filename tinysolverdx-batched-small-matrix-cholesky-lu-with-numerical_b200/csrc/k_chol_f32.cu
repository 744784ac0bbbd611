// Batched blocked Cholesky kernels (potrf / posv), float instantiations.
#include "launch.cuh"
namespace tsdx {
namespace host {
template <> int run_chol<float>(const SolveArgs<float>& a, cudaStream_t st) { return run_blk<float, true>(a, st); }
template <> int run_potrs<float>(const SolveArgs<float>& a, cudaStream_t st) { return run_trs<float, false>(a, st); }
}  // namespace host
}  // namespace tsdx
