// Uneven batched stream: one call over a ragged list of matrices with n in 1..64,
// Cholesky (posv) and LU (gesv) mixed, 0..8 right-hand sides each.
//
// No reference counterpart: TinySolverDx takes one (batch, n, n) stack of equal n
// per call, so a mixed workload is one call per (kind, n, nrhs) group.
//
// Layout (all device memory, element offsets are per-matrix and caller-chosen):
//   A    packed; matrix i (n_i x n_i, row-major) at A + aoff[i]; overwritten by its factor
//   B    packed; matrix i's right-hand sides (n_i x nrhs_i) at B + boff[i]; overwritten by X
//   piv  packed; n_i pivots of an LU matrix at piv + poff[i] (ignored for Cholesky)
//   info (count) per-matrix info
//
// Schedule. A counting sort (histogram, scan, scatter) orders the matrices by
// bucket = (kind, padded order NP in {8, 16, ..., 64}, right-hand-side class
// {<= 2, <= 8}); each bucket is cut into work units of S matrices (S = 32/G
// segments per warp for NP <= 32, as unit_size lists; or one warp per matrix when
// the tuned schedule asks for it). Seven persistent launches then drain the units
// through global atomic queues, one per order class of 8 above order 16 and one for
// n <= 16, largest orders first: each drain's warps get the shared memory of its own
// largest variant, so the smaller orders keep more warps per SM, and each drain holds
// only its class's few code variants (kind x right-hand-side class x packing). Each
// unit is the same per-matrix body (blk.cuh) as the dense kernels, so the results are
// bit-identical to them. The launches are capturable in a CUDA graph (no host
// synchronisation; scratch passed in by the caller).
#pragma once
#include "blk.cuh"

namespace tsdx {
namespace dev {

constexpr int kStreamClasses = 8;                       // NP = 8 * (class + 1)
constexpr int kStreamBuckets = 2 * kStreamClasses * 2;  // kind x class x rhs class

template <class T>
struct StreamArgs {
  T* A;
  T* B;
  int* piv;
  int* info;
  const long long* aoff;
  const long long* boff;
  const long long* poff;
  const int* n;
  const int* nrhs;
  const signed char* kind;  // 0 Cholesky (posv), 1 LU (gesv)
  int count;
  int wf;                   // write the factors back to A (and the LU pivots)
  unsigned sched;           // bit c set: bucket class c (NP 8 / 16) runs one matrix per warp
  // scratch (int): counts[K], starts[K], cursor[K], unit_start[K + 1], queue head, perm[count]
  int* scratch;
};

// Queue order: bucket 0 is the largest order, so the long units start first.
__device__ __forceinline__ int np_class(int n) {
  const int c = (n + 7) / 8 - 1;
  return c < 0 ? 0 : (c >= kStreamClasses ? kStreamClasses - 1 : c);
}
__device__ __forceinline__ int bucket_of(int kind, int n, int nrhs) {
  return ((kStreamClasses - 1 - np_class(n)) * 2 + (kind ? 1 : 0)) * 2 + (nrhs > 2 ? 1 : 0);
}
__device__ __forceinline__ int bucket_class(int b) { return kStreamClasses - 1 - (b >> 2); }
// matrices per work unit for a bucket (the dense kernels' measured packings): order
// <= 8: 8 (Cholesky, 4 lanes each) or 4 (LU); order 9..16: 4; order 17..24: 4 in
// float32, 2 in float64; order 25..32: 2; above: 1. Sched bit c (order class c =
// 0..3) asks for one matrix per warp instead.
template <class T>
__device__ __forceinline__ int unit_size(int b, unsigned sched) {
  const int c = bucket_class(b);
  const bool lu = (b >> 1) & 1;
  if (c >= 4 || ((sched >> c) & 1u)) return 1;
  if (c == 0) return lu ? 4 : 8;
  if (c == 1) return 4;
  if (c == 2) return sizeof(T) == 4 ? 4 : 2;
  return 2;
}

template <class T>
__global__ void stream_hist_kernel(StreamArgs<T> a) {
  __shared__ int h[kStreamBuckets];
  for (int t = threadIdx.x; t < kStreamBuckets; t += blockDim.x) h[t] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.count) atomicAdd(&h[bucket_of(a.kind[i], a.n[i], a.nrhs[i])], 1);
  __syncthreads();
  for (int t = threadIdx.x; t < kStreamBuckets; t += blockDim.x)
    if (h[t]) atomicAdd(&a.scratch[t], h[t]);
}

template <class T>
__global__ void stream_scan_kernel(StreamArgs<T> a) {
  if (threadIdx.x != 0) return;
  int* cnt = a.scratch;
  int* start = cnt + kStreamBuckets;
  int* cur = start + kStreamBuckets;
  int* ustart = cur + kStreamBuckets;
  int s = 0, u = 0;
  for (int b = 0; b < kStreamBuckets; ++b) {
    start[b] = s;
    cur[b] = s;
    ustart[b] = u;
    s += cnt[b];
    const int us = unit_size<T>(b, a.sched);
    u += (cnt[b] + us - 1) / us;
  }
  ustart[kStreamBuckets] = u;
  ustart[kStreamBuckets + 1] = 0;  // queue head
}

// Scatter: each block reserves one range per bucket, then places its matrices in it.
template <class T>
__global__ void stream_scatter_kernel(StreamArgs<T> a) {
  __shared__ int h[kStreamBuckets], base[kStreamBuckets];
  for (int t = threadIdx.x; t < kStreamBuckets; t += blockDim.x) h[t] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int b = 0, local = 0;
  if (i < a.count) {
    b = bucket_of(a.kind[i], a.n[i], a.nrhs[i]);
    local = atomicAdd(&h[b], 1);
  }
  __syncthreads();
  int* cur = a.scratch + 2 * kStreamBuckets;
  for (int t = threadIdx.x; t < kStreamBuckets; t += blockDim.x)
    if (h[t]) base[t] = atomicAdd(&cur[t], h[t]);
  __syncthreads();
  int* perm = a.scratch + 4 * kStreamBuckets + 2;
  if (i < a.count) perm[base[b] + local] = i;
}

template <class T, int NP, int NRHS, bool CHOL, int G>
__device__ __forceinline__ void stream_unit(unsigned char* M, const StreamArgs<T>& a, const int* perm, int first,
                                            int last, int lane) {
  Seg g;
  g.lane = lane;
  g.lsl = lane & (G - 1);
  g.segbase = (lane / G) * G;
  g.segmask = (G == 32) ? kFull : (((1u << G) - 1u) << g.segbase);
  const int idx = first + lane / G;
  MatJob<T> j;
  j.live = idx < last;
  const int m = j.live ? perm[idx] : 0;
  if (j.live) {
    // entries outside n in [1, 64], nrhs in [0, 8] are not solved: info = -1
    const int nn = a.n[m], rr = a.nrhs[m];
    if (nn < 1 || nn > NP || rr < 0 || rr > 8) {
      if ((lane & (G - 1)) == 0 && a.info) a.info[m] = -1;
      j.live = false;
    }
  }
  j.n = j.live ? a.n[m] : NP;
  j.nrhs = j.live ? a.nrhs[m] : 0;
  j.ldb = j.nrhs;
  j.b0 = 0;
  j.A = a.A + (j.live ? a.aoff[m] : 0);
  j.Aout = (j.live && a.wf) ? a.A + a.aoff[m] : nullptr;
  j.B = (j.live && a.B && j.nrhs > 0) ? a.B + a.boff[m] : nullptr;
  j.piv = (!CHOL && j.live && a.wf && a.piv) ? a.piv + a.poff[m] : nullptr;
  j.info = (j.live && a.info) ? a.info + m : nullptr;
  blk_matrix<T, NP, NRHS, CHOL, G>(M + (lane / G) * BlkCfg<T, NP, NRHS, G>::SEGB, j, g);
}

// Persistent drain of the work units of order classes CLO..CHI (one launch per class
// group, largest orders first). Every warp owns WARPB bytes of shared memory, sized for
// the largest variant of its group, so the groups of smaller orders keep more warps per
// SM. The classes' buckets are contiguous in bucket order, hence so are their units.
// The group's queue head is the bucket cursor cur[CLO]: the cursors are dead once the
// scatter has run, and the host zeroes them before the drains.
template <class T, int WARPB, int WPC, int CLO, int CHI>
__global__ void __launch_bounds__(WPC * 32, 1) stream_kernel(StreamArgs<T> a) {
  static_assert(0 <= CLO && CLO <= CHI && CHI < kStreamClasses, "class range");
  constexpr int B_LO = (kStreamClasses - 1 - CHI) * 4, B_HI = (kStreamClasses - CLO) * 4;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int ustart_s[kStreamBuckets + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int* start = a.scratch + kStreamBuckets;
  const int* cnt = a.scratch;
  const int* ustart = a.scratch + 3 * kStreamBuckets;
  int* head = a.scratch + 2 * kStreamBuckets + CLO;
  const int* perm = a.scratch + 4 * kStreamBuckets + 2;
  if (threadIdx.x <= kStreamBuckets) ustart_s[threadIdx.x] = ustart[threadIdx.x];
  __syncthreads();
  const int u0 = ustart_s[B_LO], total = ustart_s[B_HI];
  unsigned char* M = smem + warp * WARPB;
  for (;;) {
    int w = 0;
    if (lane == 0) w = u0 + atomicAdd(head, 1);
    w = __shfl_sync(kFull, w, 0);
    if (w >= total) break;
    int b = B_LO;
    while (b + 1 < B_HI && ustart_s[b + 1] <= w) ++b;
    const int us = unit_size<T>(b, a.sched);
    const int first = start[b] + (w - ustart_s[b]) * us;
    const int last = min(first + us, start[b] + cnt[b]);
    const bool one = us == 1;
    const int c = bucket_class(b);
    const bool lu = (b >> 1) & 1, wide = b & 1;
#define TSDX_SU(NP_, R_, CH_, G_) stream_unit<T, NP_, R_, CH_, G_>(M, a, perm, first, last, lane)
#define TSDX_SU_KIND(NP_, R_, G_) \
  if (lu) TSDX_SU(NP_, R_, false, G_); \
  else TSDX_SU(NP_, R_, true, G_)
#define TSDX_SU_RHS(NP_, G_) \
  if (wide) { TSDX_SU_KIND(NP_, 8, G_); } \
  else { TSDX_SU_KIND(NP_, 2, G_); }
    switch (c) {
      case 0:
        if constexpr (CLO > 0) {
        } else if (one) {
          TSDX_SU_RHS(8, 32)
        } else if (wide) {
          if (lu) TSDX_SU(8, 8, false, 8);
          else TSDX_SU(8, 8, true, 4);
        } else {
          if (lu) TSDX_SU(8, 2, false, 8);
          else TSDX_SU(8, 2, true, 4);
        }
        break;
      case 1:
        if constexpr (CLO <= 1 && CHI >= 1) {
          if (one) { TSDX_SU_RHS(16, 32) } else { TSDX_SU_RHS(16, 8) }
        }
        break;
      case 2:
        if constexpr (CLO > 2 || CHI < 2) {
        } else if (one) {
          TSDX_SU_RHS(24, 32)
        } else if constexpr (sizeof(T) == 4) {
          TSDX_SU_RHS(24, 8)
        } else {
          TSDX_SU_RHS(24, 16)
        }
        break;
      case 3:
        if constexpr (CLO <= 3 && CHI >= 3) {
          if (one) { TSDX_SU_RHS(32, 32) } else { TSDX_SU_RHS(32, 16) }
        }
        break;
      case 4:
        if constexpr (CLO <= 4 && CHI >= 4) { TSDX_SU_RHS(40, 32) }
        break;
      case 5:
        if constexpr (CLO <= 5 && CHI >= 5) { TSDX_SU_RHS(48, 32) }
        break;
      case 6:
        if constexpr (CLO <= 6 && CHI >= 6) { TSDX_SU_RHS(56, 32) }
        break;
      default:
        if constexpr (CHI >= 7) { TSDX_SU_RHS(64, 32) }
        break;
    }
#undef TSDX_SU_RHS
#undef TSDX_SU_KIND
#undef TSDX_SU
  }
}

}  // namespace dev
}  // namespace tsdx
