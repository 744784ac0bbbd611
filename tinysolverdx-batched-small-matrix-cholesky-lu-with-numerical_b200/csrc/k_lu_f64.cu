// Batched blocked LU kernels (getrf / gesv), double instantiations.
#include "launch.cuh"
namespace tsdx {
namespace host {
template <> int run_lu<double>(const SolveArgs<double>& a, cudaStream_t st) { return run_blk<double, false>(a, st); }
template <> int run_getrs<double>(const SolveArgs<double>& a, cudaStream_t st) { return run_trs<double, true>(a, st); }
}  // namespace host
}  // namespace tsdx
