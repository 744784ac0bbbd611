// Batched blocked LU kernels (getrf / gesv), float instantiations.
#include "launch.cuh"
namespace tsdx {
namespace host {
template <> int run_lu<float>(const SolveArgs<float>& a, cudaStream_t st) { return run_blk<float, false>(a, st); }
template <> int run_getrs<float>(const SolveArgs<float>& a, cudaStream_t st) { return run_trs<float, true>(a, st); }
}  // namespace host
}  // namespace tsdx
