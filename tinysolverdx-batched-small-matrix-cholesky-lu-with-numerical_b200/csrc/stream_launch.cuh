// Host side of the uneven stream (stream.cuh): counting sort into buckets + persistent
// drains (one per order class above order 16, one for n <= 16), instantiated per element type in k_stream_f32.cu /
// k_stream_f64.cu.
#pragma once
#include <cuda_runtime.h>

#include "../../include/tsdx_cuda.h"
#include "launch.cuh"
#include "stream.cuh"

namespace tsdx {
namespace host {

namespace {
constexpr int cmax(int a, int b) { return a > b ? a : b; }
// shared memory per warp of the variants of order class c (the drain's switch): one
// matrix per warp, and the packed layouts of classes 0..3
template <class T> constexpr int class_warpb(int c) {
  using dev::BlkCfg;
  switch (c) {
    case 0: return cmax(BlkCfg<T, 8, 8, 32>::WARPB, cmax(BlkCfg<T, 8, 8, 8>::WARPB, BlkCfg<T, 8, 8, 4>::WARPB));
    case 1: return cmax(BlkCfg<T, 16, 8, 32>::WARPB, BlkCfg<T, 16, 8, 8>::WARPB);
    case 2: return cmax(BlkCfg<T, 24, 8, 32>::WARPB, BlkCfg<T, 24, 8, sizeof(T) == 4 ? 8 : 16>::WARPB);
    case 3: return cmax(BlkCfg<T, 32, 8, 32>::WARPB, BlkCfg<T, 32, 8, 16>::WARPB);
    case 4: return BlkCfg<T, 40, 8, 32>::WARPB;
    case 5: return BlkCfg<T, 48, 8, 32>::WARPB;
    case 6: return BlkCfg<T, 56, 8, 32>::WARPB;
    default: return BlkCfg<T, 64, 8, 32>::WARPB;
  }
}
// shared memory per warp of a drain over classes lo..hi: the largest of their variants
template <class T> constexpr int stream_warpb(int lo, int hi) {
  int m = 0;
  for (int c = lo; c <= hi; ++c) m = cmax(m, class_warpb<T>(c));
  return m;
}

// one drain launch over order classes CLO..CHI
template <class T, int CLO, int CHI>
int launch_drain(const dev::StreamArgs<T>& a, cudaStream_t st) {
  constexpr int WARPB = stream_warpb<T>(CLO, CHI);
  constexpr int FIT = (227 * 1024) / WARPB;
  constexpr int WPC = FIT < 1 ? 1 : (FIT > 16 ? 16 : FIT);
  constexpr int SMEM = WPC * WARPB;
  auto kern = dev::stream_kernel<T, WARPB, WPC, CLO, CHI>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const int grid = grid_for(kern, SMEM, 1LL << 30, WPC * 32);
  kern<<<grid, WPC * 32, SMEM, st>>>(a);
  return 0;
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
  int rc = 0;
  cudaError_t e = cudaMemsetAsync(a.scratch, 0, dev::kStreamBuckets * sizeof(int), st);
  if (e == cudaSuccess) {
    const unsigned blocks = (unsigned)((a.count + 255) / 256);
    dev::stream_hist_kernel<T><<<blocks, 256, 0, st>>>(a);
    dev::stream_scan_kernel<T><<<1, 32, 0, st>>>(a);
    dev::stream_scatter_kernel<T><<<blocks, 256, 0, st>>>(a);
    // the bucket cursors are dead after the scatter: zero them, they are the drains' queue heads
    e = cudaMemsetAsync(a.scratch + 2 * dev::kStreamBuckets, 0, dev::kStreamClasses * sizeof(int), st);
  }
  // seven drains, largest orders first: one per order class of 8 above order 16, one for
  // n <= 16. Shared memory per warp is sized for each class, so the smaller orders keep
  // more warps per SM, and each drain carries only its class's code variants (one
  // drain over n <= 48 carried about 40 and stalled on instruction fetch).
  if (e == cudaSuccess) rc = launch_drain<T, 7, 7>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 6, 6>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 5, 5>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 4, 4>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 3, 3>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 2, 2>(a, st);
  if (e == cudaSuccess && !rc) rc = launch_drain<T, 0, 1>(a, st);
  if (e == cudaSuccess && !rc) {
    launch_counter().fetch_add(10);
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
