// Shared device helpers of the batched small-matrix kernels (sm_100a): argument
// block, element-type traits, the bit-exact arithmetic building blocks, and copy
// helpers.
//
// Bit-exactness. Every factor element receives exactly the reference's chain of
// operations (TinySolverDx kernels.hpp): LU (kernels.hpp:91-119) a_ij <-
// fma(-l_ik, u_kj, a_ij) in increasing k with l_ik = a_ik / u_kk correctly
// rounded (Markstein-corrected reciprocal below); Cholesky as the reference's
// default simd backend compiles it (kernels.hpp:57-87: fused for n <= 16, product
// rounded before the subtraction for n >= 17, sub_mul below). The pivot search
// compares keys built from |a| so that the reference's tie-breaking (strict '>',
// first maximum wins, NaN never wins unless it sits on the diagonal position) is
// reproduced exactly (seg_argmax below).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tsdx {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;

template <class T> struct KeyT;
template <> struct KeyT<double> { using U = unsigned long long; };
template <> struct KeyT<float> { using U = unsigned; };

__device__ __forceinline__ unsigned long long key_bits(double v) { return (unsigned long long)__double_as_longlong(fabs(v)); }
__device__ __forceinline__ unsigned key_bits(float v) { return __float_as_uint(fabsf(v)); }

__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// s - x*y with the product rounded first (never contracted)
__device__ __forceinline__ double sub_mul(double s, double x, double y) { return __dsub_rn(s, __dmul_rn(x, y)); }
__device__ __forceinline__ float sub_mul(float s, float x, float y) { return __fsub_rn(s, __fmul_rn(x, y)); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double sqrt_(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float sqrt_(float a) { return __fsqrt_rn(a); }

// ---- correctly rounded division by a value whose reciprocal is shared -----------
// Markstein's correction step (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990): with
// y = RN(1/b) and q = RN(a*y), the remainder e = a - b*q is exact (one FMA) and
// RN(q + e*y) = RN(a/b) as long as no intermediate underflows or overflows.
// A pivot step divides a whole column by one pivot, so y is computed once
// (__drcp_rn / __frcp_rn, IEEE round-to-nearest) and every quotient costs a
// multiply and two FMAs. A zero numerator is answered by q itself whenever q is
// not NaN: then y is finite, so b is neither zero nor NaN, and a*y is the zero
// with the sign of a XOR the sign of b (RN(1/b) keeps b's sign, also when it
// underflows), which is IEEE's a/b. This case is common, not rare: the rows that
// pad an order up to its kernel's tile are zero left of the diagonal block, so
// each pivot step divides zeros. Other operands outside the safe range
// (subnormals, huge values, Inf, NaN, a zero over a zero or a subnormal divisor)
// take the IEEE division. Checked bit-for-bit against __ddiv_rn / __fdiv_rn by
// tests/test_gpu_parity.py::test_markstein_division.
static __device__ __noinline__ double div_slow(double a, double b) { return __ddiv_rn(a, b); }
static __device__ __noinline__ float div_slow(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rcp_(double b) { return __drcp_rn(b); }
__device__ __forceinline__ float rcp_(float b) { return __frcp_rn(b); }
__device__ __forceinline__ double div_by(double a, double b, double y) {
  const double q = __dmul_rn(a, y);
  const double aq = fabs(q), aa = fabs(a);
  if (!(aq >= 0x1p-960 && aq <= 0x1p+960 && aa >= 0x1p-960 && aa <= 0x1p+960)) return (a == 0.0 && q == 0.0) ? q : div_slow(a, b);
  const double e = __fma_rn(-b, q, a);
  return __fma_rn(e, y, q);
}
__device__ __forceinline__ float div_by(float a, float b, float y) {
  const float q = __fmul_rn(a, y);
  const float aq = fabsf(q), aa = fabsf(a);
  if (!(aq >= 0x1p-100f && aq <= 0x1p+100f && aa >= 0x1p-100f && aa <= 0x1p+100f)) return (a == 0.0f && q == 0.0f) ? q : div_slow(a, b);
  const float e = __fmaf_rn(-b, q, a);
  return __fmaf_rn(e, y, q);
}

__device__ __forceinline__ void named_barrier(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// ---- argmax over a lane segment: larger key wins, ties go to the smaller position.
__device__ __forceinline__ int seg_argmax(unsigned mask, unsigned long long key, int pos, unsigned long long* kout) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(mask, hi);
  const unsigned mlo = __reduce_max_sync(mask, hi == mhi ? lo : 0u);
  const int cand = (hi == mhi && lo == mlo) ? pos : 0x7fffffff;
  *kout = ((unsigned long long)mhi << 32) | mlo;
  return __reduce_min_sync(mask, cand);
}
__device__ __forceinline__ int seg_argmax(unsigned mask, unsigned key, int pos, unsigned* kout) {
  const unsigned mk = __reduce_max_sync(mask, key);
  *kout = mk;
  return __reduce_min_sync(mask, key == mk ? pos : 0x7fffffff);
}

// Exact warp argmax: the largest key wins, ties go to the smallest position. The
// first reduction runs on the key's high word; when one lane alone holds that
// word, it is the winner and no further reduction is needed. *zero: the winning
// key is 1 (|a| = 0).
__device__ __forceinline__ int warp_argmax(unsigned long long key, int pos, bool* zero) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(kFull, hi);
  const unsigned bal = __ballot_sync(kFull, hi == mhi);
  if (__popc(bal) == 1) {  // then mhi > 0, so the key is not 1
    *zero = false;
    return __shfl_sync(kFull, pos, __ffs(bal) - 1);
  }
  const unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
  *zero = (mhi == 0u && mlo == 1u);
  return __reduce_min_sync(kFull, (hi == mhi && lo == mlo) ? pos : 0x7fffffff);
}
__device__ __forceinline__ int warp_argmax(unsigned key, int pos, bool* zero) {
  const unsigned mk = __reduce_max_sync(kFull, key);
  *zero = (mk == 1u);
  const unsigned bal = __ballot_sync(kFull, key == mk);
  if (__popc(bal) == 1) return __shfl_sync(kFull, pos, __ffs(bal) - 1);
  return __reduce_min_sync(kFull, key == mk ? pos : 0x7fffffff);
}

// The same, also returning the winner's lane: the lane whose best candidate is the
// winning (key, position).
__device__ __forceinline__ int warp_argmax_lane(unsigned long long key, int pos, bool* zero, int* wl) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(kFull, hi);
  const unsigned bal = __ballot_sync(kFull, hi == mhi);
  if (__popc(bal) == 1) {
    *zero = false;
    *wl = __ffs(bal) - 1;
    return __shfl_sync(kFull, pos, *wl);
  }
  const unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
  *zero = (mhi == 0u && mlo == 1u);
  const int bpos = __reduce_min_sync(kFull, (hi == mhi && lo == mlo) ? pos : 0x7fffffff);
  *wl = __ffs(__ballot_sync(kFull, pos == bpos)) - 1;
  return bpos;
}

// ---- cp.async (LDGSTS) staging of a global byte range into padded rows --------
template <int VEC>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (VEC == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
  else if constexpr (VEC == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Fast division of small non-negative ints by a runtime divisor d (d <= 4096,
// x < 2^19): q = umulhi(x, ceil(2^32/d)) is exact in that range.
struct FastDiv {
  unsigned d, m;
  __host__ __device__ FastDiv() : d(1), m(0) {}
  __host__ __device__ explicit FastDiv(unsigned dd) : d(dd), m((unsigned)((0x100000000ull + dd - 1) / dd)) {}
  __device__ __forceinline__ unsigned div(unsigned x) const { return d == 1 ? x : __umulhi(x, m); }
};

template <class T>
struct SolveArgs {
  T* A;            // (batch, n, n) row-major; overwritten by the factor
  T* B;            // (batch, n, ldb) row-major; columns [b0, b0 + nrhs) are solved in place
  int* piv;        // (batch, n) LU pivots, 0-based sequential (LU only)
  int* info;       // (batch) or nullptr
  long long batch;
  int n, ldb, b0, nrhs;
  FastDiv rowdiv;      // divides by the number of copy chunks per row
  const int* status;   // optional: matrices with status[m] >= 0 are skipped (no reads, no writes)
  int wf;              // 1: A <- factor and piv written (reference semantics); 0: A left untouched
};

}  // namespace dev
}  // namespace tsdx

namespace tsdx {
namespace dev {

// 16-byte shared-memory vector access (2 doubles / 4 floats).
template <class T> struct Vec16;
template <> struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ static __forceinline__ double get(const double2& v, int i) { return i == 0 ? v.x : v.y; }
  __device__ static __forceinline__ void set(double2& v, int i, double x) { if (i == 0) v.x = x; else v.y = x; }
};
template <> struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ static __forceinline__ float get(const float4& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
  __device__ static __forceinline__ void set(float4& v, int i, float x) {
    if (i == 0) v.x = x; else if (i == 1) v.y = x; else if (i == 2) v.z = x; else v.w = x;
  }
};

// Copies rows [0, rows) of a dense (rows x n) stack at g into padded staging rows
// (row stride RS bytes) with VEC-byte cp.async chunks; rc = n*sizeof(T)/VEC.
template <class T, int VEC, int RS, int BUF>
__device__ __forceinline__ void stage_in(unsigned char* stage, const char* g, int rows, int n, int rc,
                                         const FastDiv& rowdiv, const FastDiv& ndiv, int tt, int TT) {
  const int chunks = rows * rc;
  for (int e = tt; e < chunks; e += TT) {
    const int row = (int)rowdiv.div(e), ch = e - row * rc;
    const int mm = (int)ndiv.div(row), r = row - mm * n;
    cp_async<VEC>(stage + mm * BUF + r * RS + ch * VEC, g + (long long)row * n * int(sizeof(T)) + ch * VEC);
  }
  cp_async_commit();
}
template <class T, int VEC, int RS, int BUF>
__device__ __forceinline__ void stage_out(const unsigned char* stage, char* g, int rows, int n, int rc,
                                          const FastDiv& rowdiv, const FastDiv& ndiv, int tt, int TT) {
  const int chunks = rows * rc;
  for (int e = tt; e < chunks; e += TT) {
    const int row = (int)rowdiv.div(e), ch = e - row * rc;
    const int mm = (int)ndiv.div(row), r = row - mm * n;
    const unsigned char* src = stage + mm * BUF + r * RS + ch * VEC;
    char* dst = g + (long long)row * n * int(sizeof(T)) + ch * VEC;
    if constexpr (VEC == 16) *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
    else if constexpr (VEC == 8) *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(src);
    else *reinterpret_cast<unsigned*>(dst) = *reinterpret_cast<const unsigned*>(src);
  }
}

}  // namespace dev
}  // namespace tsdx
