// C-ABI shim over the REFERENCE library, compiled from the reference's own
// sources where they lie (include/tinysolverdx/*.hpp and src/runtime.cpp of
// TinySolverDx) by oracle/Makefile into oracle/_ref/libtsdx_ref.so.
//
// Test infrastructure only: the test-suite uses it to pin the C restatement in
// tsdx_oracle.c bit-for-bit, and the benchmark's CPU-baseline leg uses it to
// time the reference's own CPU backends. Nothing in the GPU product path loads it.
//
// backend codes: 0 auto, 1 naive, 2 scalar, 3 simd (tsdx::Backend, precision.hpp:33).
// precision codes: 0 fp32, 1 fp64, 2 fp16, 3 bf16 (tsdx::Precision, precision.hpp:32).
#include <cstdint>
#include <exception>

#include "tinysolverdx/tinysolverdx.hpp"

namespace {
tsdx::Backend be(int b) {
  switch (b) {
    case 1: return tsdx::Backend::Naive;
    case 2: return tsdx::Backend::Scalar;
    case 3: return tsdx::Backend::Simd;
    default: return tsdx::Backend::Auto;
  }
}
tsdx::Precision pr(int p) {
  switch (p) {
    case 0: return tsdx::Precision::FP32;
    case 2: return tsdx::Precision::FP16;
    case 3: return tsdx::Precision::BF16;
    default: return tsdx::Precision::FP64;
  }
}
template <class F> int guard(F&& f) {
  try { f(); return 0; } catch (const std::exception&) { return -1; }
}
}  // namespace

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int ref_num_threads() { return tsdx::num_threads(); }
REF_API void ref_set_num_threads(int n) { tsdx::set_num_threads(n); }
REF_API int ref_has_openmp() { return tsdx::has_openmp() ? 1 : 0; }

#define REF_TYPED(T, S)                                                                        \
  REF_API int ref_cholesky_batched_##S(T* A, int n, int64_t batch, int* info, int b) {         \
    return guard([&] { tsdx::cholesky_batched<T>(A, n, batch, info, be(b)); });               \
  }                                                                                            \
  REF_API int ref_lu_batched_##S(T* A, int n, int64_t batch, int* piv, int* info, int b) {     \
    return guard([&] { tsdx::lu_batched<T>(A, n, batch, piv, info, be(b)); });                \
  }                                                                                            \
  REF_API int ref_cholesky_solve_batched_##S(const T* L, int n, int64_t batch, T* B, int r) {  \
    return guard([&] { tsdx::cholesky_solve_batched<T>(L, n, batch, B, r); });                \
  }                                                                                            \
  REF_API int ref_lu_solve_batched_##S(const T* LU, const int* piv, int n, int64_t batch,      \
                                       T* B, int r) {                                         \
    return guard([&] { tsdx::lu_solve_batched<T>(LU, piv, n, batch, B, r); });               \
  }                                                                                            \
  REF_API int ref_posv_batched_##S(T* A, int n, int64_t batch, T* B, int r, int* info, int b) {\
    return guard([&] { tsdx::posv_batched<T>(A, n, batch, B, r, info, be(b)); });             \
  }                                                                                            \
  REF_API int ref_gesv_batched_##S(T* A, int n, int64_t batch, T* B, int r, int* piv,          \
                                   int* info, int b) {                                        \
    return guard([&] { tsdx::gesv_batched<T>(A, n, batch, B, r, piv, info, be(b)); });        \
  }                                                                                            \
  REF_API int ref_cholesky_##S(int p, T* A, int n, int64_t batch, int* info, int b) {          \
    return guard([&] { tsdx::cholesky<T>(pr(p), A, n, batch, info, be(b)); });               \
  }                                                                                            \
  REF_API int ref_lu_##S(int p, T* A, int n, int64_t batch, int* piv, int* info, int b) {      \
    return guard([&] { tsdx::lu<T>(pr(p), A, n, batch, piv, info, be(b)); });                 \
  }                                                                                            \
  REF_API int ref_cholesky_solve_##S(int p, const T* L, int n, int64_t batch, T* B, int r) {   \
    return guard([&] { tsdx::cholesky_solve<T>(pr(p), L, n, batch, B, r); });                 \
  }                                                                                            \
  REF_API int ref_lu_solve_##S(int p, const T* LU, const int* piv, int n, int64_t batch,       \
                               T* B, int r) {                                                 \
    return guard([&] { tsdx::lu_solve<T>(pr(p), LU, piv, n, batch, B, r); });                 \
  }                                                                                            \
  REF_API void ref_round_to_##S(int p, T* x, int64_t count) { tsdx::round_to<T>(pr(p), x, count); }

REF_TYPED(float, f)
REF_TYPED(double, d)

REF_API float ref_round_fp16(float x) { return tsdx::detail::round_fp16(x); }
REF_API float ref_round_bf16(float x) { return tsdx::detail::round_bf16(x); }

REF_API void ref_chol_backward_error(const double* A, const double* L, int n, int64_t batch, double* out) {
  tsdx::chol_backward_error(A, L, n, batch, out);
}
REF_API void ref_lu_backward_error(const double* A, const double* LU, const int* piv, int n, int64_t batch,
                                   double* out) {
  tsdx::lu_backward_error(A, LU, piv, n, batch, out);
}
REF_API void ref_solve_backward_error(const double* A, const double* x, const double* b, int n, int64_t batch,
                                      double* out) {
  tsdx::solve_backward_error(A, x, b, n, batch, out);
}
REF_API void ref_solve_forward_error(const double* A, const double* x, const double* b, int n, int64_t batch,
                                     double* out) {
  tsdx::solve_forward_error(A, x, b, n, batch, out);
}
REF_API void ref_reference_solve(const double* A, const double* b, int n, int64_t batch, double* x) {
  tsdx::reference_solve(A, b, n, batch, x);
}
