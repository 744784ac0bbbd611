// Emulated fp16 / bf16 factorizations and solves on the GPU: the reference's
// per-operation-rounding formats (include/tinysolverdx/precision.hpp:41-97),
// where every +, -, *, / and sqrt is computed in float and rounded to the target
// format with no wide accumulator, run by the algorithms of kernels.hpp:18-37,
// 91-119, 184-227 over those values. The reference runs these formats only on
// the CPU (batched.hpp:130-132); here backend "cuda" runs them too, one thread
// per matrix, bit-identical to the CPU path: the rounding steps below restate
// precision.hpp's (round-to-nearest-even on the bit pattern, binary16
// subnormals by a quantum of 2^-24, overflow to infinity, NaN passed through
// unchanged), and each float operation is an explicitly rounded intrinsic so
// nothing is contracted. Storage is float64 (the runtime API's buffer type);
// every stored value is exactly representable, so the float64 round trip is exact.
#pragma once
#include <cuda_runtime.h>

namespace tsdx {
namespace dev {

__device__ __forceinline__ float emu_round_fp16(float x) {
  const unsigned u = __float_as_uint(x), sign = u & 0x80000000u, a = u & 0x7fffffffu;
  if (a >= 0x7f800000u) return x;
  const float ax = __uint_as_float(a);
  if (ax >= 65520.0f) return __uint_as_float(sign | 0x7f800000u);
  if (ax < 6.103515625e-05f) {  // below the smallest normal: multiples of 2^-24
    const float q = 5.9604644775390625e-08f;
    return __uint_as_float(sign | __float_as_uint(__fmul_rn(rintf(__fdiv_rn(ax, q)), q)));
  }
  unsigned r = a + 0xfffu + ((a >> 13) & 1u);
  r &= ~0x1fffu;
  return __uint_as_float(sign | r);
}
__device__ __forceinline__ float emu_round_bf16(float x) {
  const unsigned u = __float_as_uint(x), a = u & 0x7fffffffu;
  if (a > 0x7f800000u) return x;
  unsigned r = a + 0x7fffu + ((a >> 16) & 1u);
  r &= ~0xffffu;
  return __uint_as_float((u & 0x80000000u) | r);
}

template <int FMT>
struct EmuOps {
  static __device__ __forceinline__ float R(float x) { return FMT == 0 ? emu_round_fp16(x) : emu_round_bf16(x); }
  static __device__ __forceinline__ float sub(float a, float b) { return R(__fsub_rn(a, b)); }
  static __device__ __forceinline__ float mul(float a, float b) { return R(__fmul_rn(a, b)); }
  static __device__ __forceinline__ float div(float a, float b) { return R(__fdiv_rn(a, b)); }
  static __device__ __forceinline__ float sqrt_(float a) { return R(__fsqrt_rn(a)); }
  static __device__ __forceinline__ float in(double v) { return R(__double2float_rn(v)); }
};

// a: n x n float64 storage of one matrix, rounded to the format on entry.
template <int FMT>
__global__ void emu_cholesky_kernel(double* A, int n, long long batch, int* info) {
  using E = EmuOps<FMT>;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= batch) return;
  double* a = A + m * n * n;
  for (int e = 0; e < n * n; ++e) a[e] = (double)E::in(a[e]);
  int inf = 0;
  for (int i = 0; i < n && !inf; ++i) {
    for (int j = 0; j <= i; ++j) {
      float s = (float)a[i * n + j];
      for (int k = 0; k < j; ++k) s = E::sub(s, E::mul((float)a[i * n + k], (float)a[j * n + k]));
      if (j == i) {
        if (!(s > 0.0f)) {  // early return: the upper triangle is left as it is
          inf = i + 1;
          break;
        }
        a[i * n + i] = (double)E::sqrt_(s);
      } else {
        a[i * n + j] = (double)E::div(s, (float)a[j * n + j]);
      }
    }
  }
  if (!inf)
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) a[i * n + j] = 0.0;
  if (info) info[m] = inf;
}

template <int FMT>
__global__ void emu_lu_kernel(double* A, int n, long long batch, int* piv, int* info) {
  using E = EmuOps<FMT>;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= batch) return;
  double* a = A + m * n * n;
  int* pv = piv + m * n;
  for (int e = 0; e < n * n; ++e) a[e] = (double)E::in(a[e]);
  int inf = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    float best = (float)a[k * n + k];
    best = best < 0.0f ? -best : best;
    for (int i = k + 1; i < n; ++i) {
      float v = (float)a[i * n + k];
      v = v < 0.0f ? -v : v;
      if (v > best) {
        best = v;
        p = i;
      }
    }
    pv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        const double t = a[k * n + j];
        a[k * n + j] = a[p * n + j];
        a[p * n + j] = t;
      }
    const float pk = (float)a[k * n + k];
    if (pk == 0.0f) {
      if (inf == 0) inf = k + 1;
      continue;
    }
    for (int i = k + 1; i < n; ++i) {
      const float f = E::div((float)a[i * n + k], pk);
      a[i * n + k] = (double)f;
      for (int j = k + 1; j < n; ++j) a[i * n + j] = (double)E::sub((float)a[i * n + j], E::mul(f, (float)a[k * n + j]));
    }
  }
  if (info) info[m] = inf;
}

// B (n x nrhs) <- (L L^T)^{-1} B, or with LU = (P L U): the factor is rounded on entry.
template <int FMT, bool LU>
__global__ void emu_solve_kernel(const double* F, const int* piv, int n, long long batch, double* B, int nrhs) {
  using E = EmuOps<FMT>;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= batch) return;
  const double* f = F + m * n * n;
  double* b = B + m * (long long)n * nrhs;
  auto FF = [&](int i, int k) { return E::in(f[i * n + k]); };
  for (int e = 0; e < n * nrhs; ++e) b[e] = (double)E::in(b[e]);
  if (LU) {
    const int* pv = piv + m * n;
    for (int k = 0; k < n; ++k)
      if (pv[k] != k)
        for (int r = 0; r < nrhs; ++r) {
          const double t = b[k * nrhs + r];
          b[k * nrhs + r] = b[pv[k] * nrhs + r];
          b[pv[k] * nrhs + r] = t;
        }
  }
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k)
      for (int r = 0; r < nrhs; ++r)
        b[i * nrhs + r] = (double)E::sub((float)b[i * nrhs + r], E::mul(FF(i, k), (float)b[k * nrhs + r]));
    if (!LU)
      for (int r = 0; r < nrhs; ++r) b[i * nrhs + r] = (double)E::div((float)b[i * nrhs + r], FF(i, i));
  }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k)
      for (int r = 0; r < nrhs; ++r)
        b[i * nrhs + r] =
            (double)E::sub((float)b[i * nrhs + r], E::mul(LU ? FF(i, k) : FF(k, i), (float)b[k * nrhs + r]));
    for (int r = 0; r < nrhs; ++r) b[i * nrhs + r] = (double)E::div((float)b[i * nrhs + r], FF(i, i));
  }
}

}  // namespace dev
}  // namespace tsdx
