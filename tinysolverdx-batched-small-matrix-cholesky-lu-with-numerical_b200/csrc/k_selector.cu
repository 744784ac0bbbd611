// C-ABI of the learned precision-tier selector (selector.cuh). No reference
// counterpart. All pointers are device pointers; calls are stream-ordered.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/tsdx_cuda.h"
#include "launch.cuh"
#include "selector.cuh"

#define API extern "C" __attribute__((visibility("default")))

namespace {
using namespace tsdx;
constexpr int kFeatWpc = 8;
constexpr int kFeatSmem = 0;
constexpr int kTrainSmem = (int)sizeof(dev::TrainSmem);

int finish(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    host::set_cuda_error(e, what);
    return TSDX_ERR_CUDA;
  }
  host::launch_counter().fetch_add(1);
  return TSDX_OK;
}
long long train_blocks(long long batch) { return (batch + dev::kTrainBlock - 1) / dev::kTrainBlock; }
}  // namespace

API int tsdx_cuda_selector_features_f64(const double* A, int n, int64_t batch, const signed char* kind, int kind_all,
                                        float* features, void* stream) {
  if (n < 1 || n > 64) return TSDX_ERR_N;
  if (batch < 0) return TSDX_ERR_BATCH;
  if (batch == 0) return TSDX_OK;
  if (!A || !features) return TSDX_ERR_NULL;
  auto kern = dev::features_kernel<kFeatWpc>;
  const int grid = host::grid_for(kern, kFeatSmem, (batch + kFeatWpc - 1) / kFeatWpc, kFeatWpc * 32);
  kern<<<grid, kFeatWpc * 32, kFeatSmem, static_cast<cudaStream_t>(stream)>>>(A, n, batch, kind, kind_all, features);
  return finish("features kernel");
}

API int tsdx_cuda_mlp_forward(const float* params, const float* norm, const float* features, int64_t batch,
                              float* logits, signed char* tier, void* stream) {
  if (batch < 0) return TSDX_ERR_BATCH;
  if (batch == 0) return TSDX_OK;
  if (!params || !norm || !features) return TSDX_ERR_NULL;
  const unsigned blocks = (unsigned)((batch + 127) / 128);
  dev::mlp_forward_kernel<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(params, norm, features, batch,
                                                                                 logits, tier);
  return finish("mlp forward kernel");
}

API int64_t tsdx_cuda_mlp_scratch_bytes(int64_t batch) {
  return batch <= 0 ? 0 : train_blocks(batch) * (dev::kParams + 1) * (int64_t)sizeof(float);
}

API int tsdx_cuda_mlp_grad(const float* params, const float* norm, const float* features, const signed char* label,
                           const float* class_weight, int64_t batch, float* grad, float* loss, void* scratch,
                           int64_t scratch_bytes, void* stream) {
  if (batch <= 0) return TSDX_ERR_BATCH;
  if (!params || !norm || !features || !label || !grad || !scratch) return TSDX_ERR_NULL;
  if (scratch_bytes < tsdx_cuda_mlp_scratch_bytes(batch)) return TSDX_ERR_NULL;
  const long long blocks = train_blocks(batch);
  if (blocks > 0x7fffffffLL) return TSDX_ERR_BATCH;
  auto st = static_cast<cudaStream_t>(stream);
  if (int rc = host::prepare(dev::mlp_train_kernel, kTrainSmem)) return rc;
  float* part = static_cast<float*>(scratch);
  dev::mlp_train_kernel<<<(unsigned)blocks, dev::kTrainThreads, kTrainSmem, st>>>(params, norm, features, label,
                                                                                class_weight, batch, part);
  if (int rc = finish("mlp train kernel")) return rc;
  dev::grad_reduce_kernel<<<(dev::kParams + 1 + 255) / 256, 256, 0, st>>>(part, (int)blocks, grad, loss);
  return finish("gradient reduce kernel");
}

API int tsdx_cuda_adam_step(float* params, const float* grad, float* m, float* v, int64_t count, float lr,
                            float beta1, float beta2, float eps, int step, void* stream) {
  if (count < 0 || step < 1) return TSDX_ERR_BATCH;
  if (count == 0) return TSDX_OK;
  if (!params || !grad || !m || !v) return TSDX_ERR_NULL;
  const float c1 = (float)(1.0 - std::pow((double)beta1, step));
  const float c2 = (float)(1.0 - std::pow((double)beta2, step));
  dev::adam_kernel<<<(unsigned)((count + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grad, m, v, count, lr, beta1, beta2, eps, c1, c2);
  return finish("adam kernel");
}
