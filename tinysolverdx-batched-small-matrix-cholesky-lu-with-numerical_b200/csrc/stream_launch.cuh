// Host side of the uneven stream (stream.cuh): counting sort into buckets + one
// persistent drain, instantiated per element type in k_stream_f32.cu / k_stream_f64.cu.
#pragma once
#include <cuda_runtime.h>

#include "../../include/tsdx_cuda.h"
#include "launch.cuh"
#include "stream.cuh"

namespace tsdx {
namespace host {

namespace {
constexpr int cmax(int a, int b) { return a > b ? a : b; }
// shared memory per warp: the largest of the variants the drain can run
template <class T> constexpr int stream_warpb() {
  using dev::BlkCfg;
  constexpr int w[] = {BlkCfg<T, 8, 8>::WARPB,  BlkCfg<T, 8, 8, 32>::WARPB, BlkCfg<T, 16, 8>::WARPB,
                       BlkCfg<T, 16, 8, 32>::WARPB, BlkCfg<T, 24, 8>::WARPB, BlkCfg<T, 32, 8>::WARPB,
                       BlkCfg<T, 24, 8, 16>::WARPB, BlkCfg<T, 32, 8, 16>::WARPB, BlkCfg<T, 16, 8, 8>::WARPB,
                       BlkCfg<T, 8, 8, 4>::WARPB, BlkCfg<T, 24, 8, 8>::WARPB,
                       BlkCfg<T, 40, 8>::WARPB, BlkCfg<T, 48, 8>::WARPB, BlkCfg<T, 56, 8>::WARPB,
                       BlkCfg<T, 64, 8>::WARPB};
  int m = 0;
  for (int v : w) m = cmax(m, v);
  return m;
}
}  // namespace

constexpr long long stream_scratch_bytes_of(long long count) { return (4LL * dev::kStreamBuckets + 2 + count) * 4; }

template <class T>
int run_stream(dev::StreamArgs<T> a, void* scratch, long long scratch_bytes, cudaStream_t st) {
  if (a.count == 0) return 0;
  const long long need = stream_scratch_bytes_of(a.count);
  bool own = false;
  if (!scratch) {
    const cudaError_t e = cudaMallocAsync(&scratch, need, st);
    if (e != cudaSuccess) { set_cuda_error(e, "cudaMallocAsync"); return -5; }
    own = true;
  } else if (scratch_bytes < need) {
    return -3;
  }
  a.scratch = static_cast<int*>(scratch);
  constexpr int WARPB = stream_warpb<T>();
  constexpr int FIT = (227 * 1024) / WARPB;
  constexpr int WPC = FIT < 1 ? 1 : (FIT > 16 ? 16 : FIT);
  constexpr int SMEM = WPC * WARPB;
  auto kern = dev::stream_kernel<T, WARPB, WPC>;
  int rc = prepare(kern, SMEM);
  cudaError_t e = cudaSuccess;
  if (!rc) e = cudaMemsetAsync(a.scratch, 0, dev::kStreamBuckets * sizeof(int), st);
  if (!rc && e == cudaSuccess) {
    const unsigned blocks = (unsigned)((a.count + 255) / 256);
    dev::stream_hist_kernel<T><<<blocks, 256, 0, st>>>(a);
    dev::stream_scan_kernel<T><<<1, 32, 0, st>>>(a);
    dev::stream_scatter_kernel<T><<<blocks, 256, 0, st>>>(a);
    const int grid = grid_for(kern, SMEM, 1LL << 30, WPC * 32);
    kern<<<grid, WPC * 32, SMEM, st>>>(a);
    launch_counter().fetch_add(4);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) { set_cuda_error(e, "stream launch"); rc = -5; }
  if (own) {
    const cudaError_t f = cudaFreeAsync(scratch, st);
    if (f != cudaSuccess && !rc) { set_cuda_error(f, "cudaFreeAsync"); rc = -5; }
  }
  return rc;
}

}  // namespace host
}  // namespace tsdx
