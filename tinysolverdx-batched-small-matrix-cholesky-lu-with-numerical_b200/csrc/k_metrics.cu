// C-ABI of the GPU error metrics (metrics.cuh). Device pointers, stream-ordered.
#include <cuda_runtime.h>

#include "../../include/tsdx_cuda.h"
#include "launch.cuh"
#include "metrics.cuh"

#define API extern "C" __attribute__((visibility("default")))

namespace {
using namespace tsdx;
constexpr int kWpc = 6;
constexpr int kFactorSmem = kWpc * (64 * dev::kMetStride * (int)sizeof(double) + 64 * (int)sizeof(int));

int finish(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    host::set_cuda_error(e, what);
    return TSDX_ERR_CUDA;
  }
  host::launch_counter().fetch_add(1);
  return TSDX_OK;
}

int check(int n, int64_t batch) {
  if (n < 1 || n > 64) return TSDX_ERR_N;
  if (batch < 0) return TSDX_ERR_BATCH;
  return TSDX_OK;
}

template <bool CHOL>
int factor_metric(const double* A, const double* F, const int* piv, int n, int64_t batch, double* out, void* st) {
  if (int rc = check(n, batch)) return rc;
  if (batch == 0) return TSDX_OK;
  if (!A || !F || !out || (!CHOL && !piv)) return TSDX_ERR_NULL;
  auto kern = dev::factor_bwd_kernel<kWpc, CHOL>;
  if (int rc = host::prepare(kern, kFactorSmem)) return rc;
  const int grid = host::grid_for(kern, kFactorSmem, (batch + kWpc - 1) / kWpc, kWpc * 32);
  kern<<<grid, kWpc * 32, kFactorSmem, static_cast<cudaStream_t>(st)>>>(A, F, piv, n, batch, out);
  return finish(CHOL ? "cholesky backward error kernel" : "lu backward error kernel");
}
}  // namespace

API int tsdx_cuda_solve_backward_error_f64(const double* A, const double* x, const double* b, int n, int64_t batch,
                                           double* out, void* stream) {
  if (int rc = check(n, batch)) return rc;
  if (batch == 0) return TSDX_OK;
  if (!A || !x || !b || !out) return TSDX_ERR_NULL;
  auto kern = dev::solve_bwd_kernel<8>;
  const int grid = host::grid_for(kern, 0, (batch + 7) / 8, 256);
  kern<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(A, x, b, n, batch, out);
  return finish("solve backward error kernel");
}

API int tsdx_cuda_lu_backward_error_f64(const double* A, const double* LU, const int* piv, int n, int64_t batch,
                                        double* out, void* stream) {
  return factor_metric<false>(A, LU, piv, n, batch, out, stream);
}

API int tsdx_cuda_chol_backward_error_f64(const double* A, const double* L, int n, int64_t batch, double* out,
                                          void* stream) {
  return factor_metric<true>(A, L, nullptr, n, batch, out, stream);
}
