// Triangular solves from an existing factor: potrs (L L^T x = b) and getrs
// (P L U x = b) — TinySolverDx kernels.hpp:184-227 driven by batched.hpp:248-268
// (which the reference always runs on the CPU; here they run on the GPU).
//
// One warp per matrix: the factor is staged to shared memory with cp.async, the
// right-hand sides live in registers (lane l owns rows l and l + 32). The forward
// substitution keeps the reference's chain (increasing k, fused multiply-add, and
// for Cholesky the division by l_ii); the backward substitution is column-oriented
// and multiplies by the reciprocal of the diagonal, so X agrees with the
// reference to rounding.
#pragma once
#include "common.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP>
struct SolveSmem {
  static constexpr int RS = NP * int(sizeof(T)) + 16;
  static constexpr int WARP = NP * RS + 64 * 4;  // staged factor + permutation
  static constexpr int CTA = 4 * WARP;
};

// LU == true: getrs with pivots; LU == false: potrs.
template <class T, int NP, int NRHS, bool LU>
__global__ void __launch_bounds__(128) trs_kernel(SolveArgs<T> p, FastDiv ndiv, int vec) {
  using SM = SolveSmem<T, NP>;
  constexpr int MR = (NP + 31) / 32;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* stage = smem + warp * SM::WARP;
  int* perm = reinterpret_cast<int*>(stage + NP * SM::RS);
  const int n = p.n;
  const long long nn = (long long)n * n;
  const int rc = n * int(sizeof(T)) / vec;
  const long long nw = (long long)gridDim.x * 4;

  for (long long m = (long long)blockIdx.x * 4 + warp; m < p.batch; m += nw) {
    const char* g = reinterpret_cast<const char*>(p.A + m * nn);
    if (vec == 16) stage_in<T, 16, SM::RS, SM::WARP>(stage, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
    else if (vec == 8) stage_in<T, 8, SM::RS, SM::WARP>(stage, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
    else stage_in<T, 4, SM::RS, SM::WARP>(stage, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
    if (LU) {
      for (int i = lane; i < n; i += 32) perm[i] = i;
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < n; ++k) {  // kernels.hpp:207-213: swaps applied in k order
          int q = p.piv[m * n + k];
          q = (q < 0 || q >= n) ? k : q;  // out-of-range pivots are ignored, never dereferenced
          const int t = perm[k]; perm[k] = perm[q]; perm[q] = t;
        }
    }
    cp_async_wait<0>();
    __syncwarp();
    auto at = [&](int r, int c) -> T { return *reinterpret_cast<const T*>(stage + r * SM::RS + c * int(sizeof(T))); };

    T b[MR][NRHS];
    const long long bbase = m * (long long)n * p.ldb + p.b0;
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      const int src = (r < n) ? (LU ? perm[r] : r) : 0;
#pragma unroll
      for (int c = 0; c < NRHS; ++c) b[s][c] = (r < n && c < p.nrhs) ? p.B[bbase + (long long)src * p.ldb + c] : T(0);
    }
    // forward: L y = P b
    for (int k = 0; k < n; ++k) {
      const int ks = k >> 5, kl = k & 31;
      const T lkk = LU ? T(1) : at(k, k);
#pragma unroll
      for (int c = 0; c < NRHS; ++c) {
        T v = b[0][c];
        if (MR > 1 && ks == 1) v = b[MR - 1][c];
        T y = __shfl_sync(kFull, v, kl);
        if (!LU) y = div_(y, lkk);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          const T lrk = (r > k && r < n) ? at(r, k) : T(0);
          b[s][c] = (r == k) ? y : ((r > k && r < n) ? fma_(-lrk, y, b[s][c]) : b[s][c]);
        }
      }
    }
    // backward: U x = y (LU) or L^T x = y (Cholesky)
    for (int k = n - 1; k >= 0; --k) {
      const int ks = k >> 5, kl = k & 31;
      const T rinv = rcp_(at(k, k));
      T ck[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        ck[s] = (r < k) ? (LU ? at(r, k) : at(k, r)) : T(0);
      }
#pragma unroll
      for (int c = 0; c < NRHS; ++c) {
        T v = b[0][c];
        if (MR > 1 && ks == 1) v = b[MR - 1][c];
        const T x = __shfl_sync(kFull, v * rinv, kl);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          b[s][c] = (r == k) ? x : ((r < k) ? fma_(-ck[s], x, b[s][c]) : b[s][c]);
        }
      }
    }
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      if (r >= n) continue;
#pragma unroll
      for (int c = 0; c < NRHS; ++c)
        if (c < p.nrhs) p.B[bbase + (long long)r * p.ldb + c] = b[s][c];
    }
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace tsdx
