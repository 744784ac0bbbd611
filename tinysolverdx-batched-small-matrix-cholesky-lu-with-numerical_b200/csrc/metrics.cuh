// Error metrics on the GPU: the reference's long-double ground-truth metrics
// (src/runtime.cpp:194-242) restated in double-double arithmetic, one warp per
// matrix, so that error reports over whole batches need no host round trip.
//
//   chol_backward_error   ||A - L L^T||_F / ||A||_F                  (runtime.cpp:194-206)
//   lu_backward_error     ||P A - L U||_F / ||A||_F, P from the pivots (runtime.cpp:208-228)
//   solve_backward_error  ||b - A x||_2 / (||A||_F ||x||_2 + ||b||_2) (runtime.cpp:230-242)
//
// Double-double (a value is an unevaluated sum hi + lo, |lo| <= ulp(hi)/2) carries
// about 106 significand bits, more than the reference's x87 long double (64), so
// the sums of products here are at least as accurate as the reference's. The
// building blocks are the published error-free transformations: TwoSum (Knuth,
// TAOCP vol. 2, 4.2.2), TwoProduct with a fused multiply-add, and the
// double-double additions of Hida, Li and Bailey ("Algorithms for quad-double
// precision floating point arithmetic", ARITH-15, 2001).
#pragma once
#include <cuda_runtime.h>

namespace tsdx {
namespace dev {

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return {s, e};
}
__device__ __forceinline__ DD fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = __dadd_rn(a, b);
  return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo = __dadd_rn(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = __dadd_rn(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}
// a + x*y with the product taken exactly (TwoProduct by FMA)
__device__ __forceinline__ DD dd_fma(DD a, double x, double y) {
  const double p = __dmul_rn(x, y);
  const double e = __fma_rn(x, y, -p);
  return dd_add(a, DD{p, e});
}
__device__ __forceinline__ DD dd_sqr(DD a) {
  const double p = __dmul_rn(a.hi, a.hi);
  double e = __fma_rn(a.hi, a.hi, -p);
  e = __fma_rn(__dmul_rn(2.0, a.hi), a.lo, e);
  return fast_two_sum(p, e);
}
__device__ __forceinline__ DD dd_neg(DD a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ DD dd_warp_sum(DD v) {
  for (int o = 16; o > 0; o >>= 1) {
    DD w;
    w.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
    w.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
    v = dd_add(v, w);
  }
  return v;
}
__device__ __forceinline__ double dd_sqrt(DD a) { return sqrt(__dadd_rn(a.hi, a.lo)); }

constexpr int kMetStride = 65;  // doubles per staged factor row (n <= 64)

// ||b - A x|| / (||A||_F ||x|| + ||b||); lane i owns rows i and i + 32.
template <int WPC>
__global__ void __launch_bounds__(WPC * 32) solve_bwd_kernel(const double* __restrict__ A, const double* __restrict__ x,
                                                             const double* __restrict__ b, int n, long long batch,
                                                             double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (long long m = (long long)blockIdx.x * WPC + warp; m < batch; m += (long long)gridDim.x * WPC) {
    const double* a = A + m * n * n;
    const double* xv = x + m * n;
    const double* rhs = b + m * n;
    DD num{0, 0}, fa{0, 0}, fx{0, 0}, fb{0, 0};
    for (int s = 0; s < 2; ++s) {
      const int i = lane + 32 * s;
      if (i < n) {
        DD r{rhs[i], 0};
        const double* row = a + (long long)i * n;
        for (int j = 0; j < n; ++j) {
          const double v = row[j];
          r = dd_fma(r, -v, xv[j]);
          fa = dd_fma(fa, v, v);
        }
        num = dd_add(num, dd_sqr(r));
        fx = dd_fma(fx, xv[i], xv[i]);
        fb = dd_fma(fb, rhs[i], rhs[i]);
      }
    }
    num = dd_warp_sum(num);
    fa = dd_warp_sum(fa);
    fx = dd_warp_sum(fx);
    fb = dd_warp_sum(fb);
    if (lane == 0) out[m] = dd_sqrt(num) / (dd_sqrt(fa) * dd_sqrt(fx) + dd_sqrt(fb));
  }
}

// ||P A - L U||_F / ||A||_F (LU packed, unit L) or ||A - L L^T||_F / ||A||_F: the
// factor is staged in shared memory, lane i owns rows i and i + 32 of the product.
template <int WPC, bool CHOL>
__global__ void __launch_bounds__(WPC * 32) factor_bwd_kernel(const double* __restrict__ A,
                                                              const double* __restrict__ F, const int* __restrict__ piv,
                                                              int n, long long batch, double* out) {
  extern __shared__ __align__(16) double msm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* S = msm + warp * 64 * kMetStride;
  int* perm = reinterpret_cast<int*>(msm + WPC * 64 * kMetStride) + warp * 64;
  for (long long m = (long long)blockIdx.x * WPC + warp; m < batch; m += (long long)gridDim.x * WPC) {
    const double* a = A + m * n * n;
    const double* f = F + m * n * n;
    for (int r = 0; r < n; ++r)
      for (int c = lane; c < n; c += 32) S[r * kMetStride + c] = f[(long long)r * n + c];
    if (!CHOL && lane == 0) {
      // row i of P A is row perm[i] of A (the sequential swaps of the pivots)
      for (int i = 0; i < n; ++i) perm[i] = i;
      const int* pv = piv + m * n;
      for (int k = 0; k < n; ++k) {
        const int p = pv[k];
        if (p >= 0 && p < n) {
          const int t = perm[k];
          perm[k] = perm[p];
          perm[p] = t;
        }
      }
    }
    __syncwarp();
    DD num{0, 0}, fa{0, 0};
    for (int s = 0; s < 2; ++s) {
      const int i = lane + 32 * s;
      if (i >= n) continue;
      const double* arow = a + (long long)(CHOL ? i : perm[i]) * n;
      for (int j = 0; j < n; ++j) {
        DD acc{0, 0};
        const int kmax = i < j ? i : j;
        for (int k = 0; k <= kmax; ++k) {
          if (CHOL) {
            acc = dd_fma(acc, S[i * kMetStride + k], S[j * kMetStride + k]);
          } else {
            const double lik = (k == i) ? 1.0 : S[i * kMetStride + k];
            acc = dd_fma(acc, lik, S[k * kMetStride + j]);
          }
        }
        const double av = arow[j];
        const DD d = dd_add(DD{av, 0}, dd_neg(acc));
        num = dd_add(num, dd_sqr(d));
        fa = dd_fma(fa, av, av);
      }
    }
    num = dd_warp_sum(num);
    fa = dd_warp_sum(fa);
    if (lane == 0) out[m] = dd_sqrt(num) / dd_sqrt(fa);
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace tsdx
