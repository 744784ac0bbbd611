// Drop-in C++ API of the batched solver: the typed batch drivers of TinySolverDx
// (include/tinysolverdx/batched.hpp:121-280), its runtime-precision entry points,
// long-double metrics and thread control (include/tinysolverdx/tinysolverdx.hpp:11-32),
// with the same names, argument meaning, layouts and exceptions.
//
// Backend::Cuda runs on the B200 through the C-ABI of include/tsdx_cuda.h (the
// solves and the one-shot drivers included, which the reference always runs on
// the CPU: batched.hpp:249, :260). The CPU backends (Naive, Scalar, Simd; Auto
// = Simd, scalar LU for n >= 25, batched.hpp:187) are kept because a drop-in
// must accept every backend the reference accepts; they reproduce the
// reference's results bit for bit, including its compiled contraction pattern
// (Cholesky: fused for the compile-time sizes n <= 16 of the simd tile, separate
// product and subtraction for n >= 17; the scalar dot product in 16-byte groups).
// Nothing here falls back silently: Backend::Cuda without a device throws
// std::runtime_error, exactly like the reference built without CUDA
// (batched.hpp:132). The emulated fp16/bf16 formats, which the reference refuses
// on Backend::Cuda (batched.hpp:130-132), run on the GPU here, bit-identical to
// the CPU path (tsdx_cuda_emu_*_host).
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "tsdx_cuda.h"

namespace tsdx {

enum class Precision { FP32, FP64, FP16, BF16 };
enum class Backend { Auto, Naive, Scalar, Simd, Cuda };

constexpr int kMinN = 1;
constexpr int kMaxN = 64;

// ------------------------------------------------------------- thread control
namespace detail {
inline int env_threads() {
  if (const char* e = std::getenv("TSDX_NUM_THREADS")) {
    const int v = std::atoi(e);
    if (v > 0) return v;
  }
  const unsigned h = std::thread::hardware_concurrency();
  return h ? static_cast<int>(h) : 1;
}
inline std::atomic<int>& thread_count() {
  static std::atomic<int> t{0};
  return t;
}
}  // namespace detail

inline int num_threads() {
  int t = detail::thread_count().load();
  if (t <= 0) { t = detail::env_threads(); detail::thread_count() = t; }
  return t;
}
inline void set_num_threads(int n) { detail::thread_count() = n > 0 ? n : detail::env_threads(); }
inline bool has_openmp() { return false; }  // a std::thread pool drives the CPU backends

inline void parallel_for(std::int64_t n_chunks, const std::function<void(std::int64_t)>& f) {
  const int nt = static_cast<int>(std::min<std::int64_t>(num_threads(), n_chunks));
  if (nt <= 1) { for (std::int64_t c = 0; c < n_chunks; ++c) f(c); return; }
  std::atomic<std::int64_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] { for (std::int64_t c; (c = next.fetch_add(1)) < n_chunks;) f(c); });
  for (auto& th : pool) th.join();
}

inline bool has_cuda() { return tsdx_cuda_available() != 0; }

// --------------------------------------------------------- precision helpers
namespace detail {
inline std::uint32_t f2u(float x) { std::uint32_t u; std::memcpy(&u, &x, 4); return u; }
inline float u2f(std::uint32_t u) { float x; std::memcpy(&x, &u, 4); return x; }
// binary16 round-to-nearest-even with subnormals and overflow to inf (precision.hpp:41-55 semantics)
inline float round_fp16(float x) {
  const std::uint32_t u = f2u(x), sign = u & 0x80000000u, a = u & 0x7fffffffu;
  if (a >= 0x7f800000u) return x;
  const float ax = u2f(a);
  if (ax >= 65520.0f) return u2f(sign | 0x7f800000u);
  if (ax < 6.103515625e-05f) return u2f(sign | f2u(std::nearbyint(ax * 16777216.0f) / 16777216.0f));
  std::uint32_t r = a + 0xfffu + ((a >> 13) & 1u);
  return u2f(sign | (r & ~0x1fffu));
}
// bfloat16 round-to-nearest-even; NaN passes through (precision.hpp:58-65 semantics)
inline float round_bf16(float x) {
  const std::uint32_t u = f2u(x), a = u & 0x7fffffffu;
  if (a > 0x7f800000u) return x;
  const std::uint32_t r = (a + 0x7fffu + ((a >> 16) & 1u)) & ~0xffffu;
  return u2f((u & 0x80000000u) | r);
}
}  // namespace detail

enum class EmuFormat { Half, BFloat16 };
// A float that always holds a value of the target format; every operation rounds.
template <EmuFormat F>
struct Emu {
  float v = 0.0f;
  static float round(float x) { return F == EmuFormat::Half ? detail::round_fp16(x) : detail::round_bf16(x); }
  Emu() = default;
  explicit Emu(float x) : v(round(x)) {}
  explicit Emu(double x) : v(round(static_cast<float>(x))) {}
  explicit Emu(int x) : v(round(static_cast<float>(x))) {}
  friend Emu operator+(Emu a, Emu b) { return Emu(a.v + b.v); }
  friend Emu operator-(Emu a, Emu b) { return Emu(a.v - b.v); }
  friend Emu operator*(Emu a, Emu b) { return Emu(a.v * b.v); }
  friend Emu operator/(Emu a, Emu b) { return Emu(a.v / b.v); }
  friend Emu operator-(Emu a) { Emu r; r.v = -a.v; return r; }
  friend bool operator>(Emu a, Emu b) { return a.v > b.v; }
  friend bool operator<(Emu a, Emu b) { return a.v < b.v; }
  friend bool operator==(Emu a, Emu b) { return a.v == b.v; }
};
using Half = Emu<EmuFormat::Half>;
using BFloat16 = Emu<EmuFormat::BFloat16>;

template <class T> struct is_native : std::integral_constant<bool, std::is_same<T, float>::value || std::is_same<T, double>::value> {};

inline double unit_roundoff(Precision p) {
  switch (p) {
    case Precision::FP32: return std::ldexp(1.0, -24);
    case Precision::FP64: return std::ldexp(1.0, -53);
    case Precision::FP16: return std::ldexp(1.0, -11);
    case Precision::BF16: return std::ldexp(1.0, -8);
  }
  return 0.0;
}

namespace detail {
// a - x*y: one fused operation, or a rounded product then a subtraction
template <class T> inline T msub(T a, T x, T y, bool fused) {
  if constexpr (is_native<T>::value) return fused ? std::fma(-x, y, a) : a - static_cast<T>(x * y);
  else return a - x * y;
}
template <class T> inline T tsqrt(T x) {
  if constexpr (is_native<T>::value) return std::sqrt(x);
  else return T(std::sqrt(x.v));
}
template <class T> inline T tabs(T x) { return x < T(0) ? -x : x; }

// ---- per-matrix CPU kernels (Backend::Naive / Scalar / Simd) ----------------
// Right-looking column Cholesky (naive); all products fused.
template <class T> int chol_naive(T* a, int n) {
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k)
      for (int i = j; i < n; ++i) a[i * n + j] = msub(a[i * n + j], a[i * n + k], a[j * n + k], true);
    if (!(a[j * n + j] > T(0))) return j + 1;
    const T d = tsqrt(a[j * n + j]);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) a[i * n + j] = a[i * n + j] / d;
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) a[i * n + j] = T(0);
  return 0;
}
// Left-looking row Cholesky. group: products in complete groups of `group` terms
// are rounded separately, the tail is fused (group >= n: all fused).
template <class T> int chol_row(T* a, int n, int group, bool tile) {
  int info = 0;
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j <= i; ++j) {
      T s = a[i * n + j];
      const int kv = group >= 64 ? 0 : j / group * group;
      for (int k = 0; k < j; ++k) s = msub(s, a[i * n + k], a[j * n + k], k >= kv);
      if (j == i) {
        const bool bad = !(s > T(0));
        if (bad) {
          if (!tile) return i + 1;
          if (info == 0) info = i + 1;
          s = T(1);
        }
        a[i * n + i] = tsqrt(s);
      } else {
        a[i * n + j] = s / a[j * n + j];
      }
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) a[i * n + j] = T(0);
  return info;
}
// Right-looking GEPP. tile: a zero pivot divides by 1 and keeps eliminating (simd);
// otherwise the column is skipped (scalar). Ties go to the first maximum; NaN never wins.
template <class T> int lu_gepp(T* a, int n, int* piv, bool tile, bool naive) {
  int info = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    T best = tabs(a[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      const T v = tabs(a[i * n + k]);
      if (naive ? (v > tabs(a[p * n + k])) : (v > best)) { best = v; p = i; }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
    const T pk = a[k * n + k];
    const bool zero = (pk == T(0));
    if (zero && info == 0) info = k + 1;
    if (zero && !tile) continue;
    const T d = zero ? T(1) : pk;
    for (int i = k + 1; i < n; ++i) {
      const T f = a[i * n + k] / d;
      a[i * n + k] = f;
      for (int j = k + 1; j < n; ++j) a[i * n + j] = msub(a[i * n + j], f, a[k * n + j], true);
    }
  }
  return info;
}
template <class T> void chol_solve(const T* L, int n, T* B, int r) {
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k)
      for (int c = 0; c < r; ++c) B[i * r + c] = msub(B[i * r + c], L[i * n + k], B[k * r + c], true);
    for (int c = 0; c < r; ++c) B[i * r + c] = B[i * r + c] / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k)
      for (int c = 0; c < r; ++c) B[i * r + c] = msub(B[i * r + c], L[k * n + i], B[k * r + c], true);
    for (int c = 0; c < r; ++c) B[i * r + c] = B[i * r + c] / L[i * n + i];
  }
}
template <class T> void lu_solve(const T* LU, const int* piv, int n, T* B, int r) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k)
      for (int c = 0; c < r; ++c) std::swap(B[k * r + c], B[piv[k] * r + c]);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < i; ++k)
      for (int c = 0; c < r; ++c) B[i * r + c] = msub(B[i * r + c], LU[i * n + k], B[k * r + c], true);
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k)
      for (int c = 0; c < r; ++c) B[i * r + c] = msub(B[i * r + c], LU[i * n + k], B[k * r + c], true);
    for (int c = 0; c < r; ++c) B[i * r + c] = B[i * r + c] / LU[i * n + i];
  }
}

inline void check_dims(int n, std::int64_t batch) {
  if (n < kMinN || n > kMaxN)
    throw std::invalid_argument("matrix size n=" + std::to_string(n) + " outside supported range [1, 64]");
  if (batch < 0) throw std::invalid_argument("negative batch");
}
inline void check_cuda(int rc) {
  if (rc == TSDX_OK) return;
  if (rc == TSDX_ERR_CUDA) throw std::runtime_error(std::string("CUDA backend: ") + tsdx_cuda_last_error());
  if (rc == TSDX_ERR_NODEV) throw std::runtime_error("CUDA backend unavailable: no device");
  throw std::invalid_argument("CUDA backend rejected the arguments (code " + std::to_string(rc) + ")");
}
template <class T> Backend resolve(Backend b) {
  if (b == Backend::Auto || (b == Backend::Simd && !is_native<T>::value))
    return is_native<T>::value ? Backend::Simd : Backend::Scalar;
  return b;
}
inline std::int64_t chunk(int n) { return std::max<std::int64_t>(1, 32768 / (std::int64_t(n) * n)); }
template <class F> void for_batch(std::int64_t batch, int n, F&& f) {
  const std::int64_t cs = chunk(n);
  parallel_for((batch + cs - 1) / cs, [&](std::int64_t c) {
    const std::int64_t e = std::min(batch, (c + 1) * cs);
    for (std::int64_t b = c * cs; b < e; ++b) f(b);
  });
}
}  // namespace detail

// ------------------------------------------------------- typed batch drivers
template <class T>
void cholesky_batched(T* A, int n, std::int64_t batch, int* info, Backend backend = Backend::Auto) {
  detail::check_dims(n, batch);
  const Backend be = detail::resolve<T>(backend);
  if (batch == 0) return;
  if (be == Backend::Cuda) {
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_cholesky_batched_host_f64(A, n, batch, info));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_cholesky_batched_host_f32(A, n, batch, info));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  const std::int64_t nn = std::int64_t(n) * n;
  // compiled contraction of the reference: simd tile fused for n <= 16; scalar in 16-byte groups
  const int group = (sizeof(T) == 8 && n == 3) ? 64 : int(16 / (is_native<T>::value ? sizeof(T) : 16));
  detail::for_batch(batch, n, [&](std::int64_t b) {
    int r;
    if (be == Backend::Naive) r = detail::chol_naive(A + b * nn, n);
    else if (be == Backend::Scalar) r = detail::chol_row(A + b * nn, n, is_native<T>::value ? group : 64, false);
    else r = detail::chol_row(A + b * nn, n, n <= 16 ? 64 : 1, true);
    if (info) info[b] = r;
  });
}

template <class T>
void lu_batched(T* A, int n, std::int64_t batch, int* piv, int* info, Backend backend = Backend::Auto) {
  detail::check_dims(n, batch);
  if (!piv) throw std::invalid_argument("piv must not be null");
  if (backend == Backend::Auto && n >= 25) backend = Backend::Scalar;
  const Backend be = detail::resolve<T>(backend);
  if (batch == 0) return;
  if (be == Backend::Cuda) {
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_lu_batched_host_f64(A, n, batch, piv, info));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_lu_batched_host_f32(A, n, batch, piv, info));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  const std::int64_t nn = std::int64_t(n) * n;
  detail::for_batch(batch, n, [&](std::int64_t b) {
    const int r = detail::lu_gepp(A + b * nn, n, piv + b * n, be == Backend::Simd, be == Backend::Naive);
    if (info) info[b] = r;
  });
}

template <class T>
void cholesky_solve_batched(const T* L, int n, std::int64_t batch, T* B, int nrhs, Backend backend = Backend::Auto) {
  detail::check_dims(n, batch);
  if (batch == 0 || nrhs == 0) return;
  if (backend == Backend::Cuda) {
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_cholesky_solve_batched_host_f64(L, n, batch, B, nrhs));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_cholesky_solve_batched_host_f32(L, n, batch, B, nrhs));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  const std::int64_t nn = std::int64_t(n) * n, bn = std::int64_t(n) * nrhs;
  detail::for_batch(batch, n, [&](std::int64_t b) { detail::chol_solve(L + b * nn, n, B + b * bn, nrhs); });
}

template <class T>
void lu_solve_batched(const T* LU, const int* piv, int n, std::int64_t batch, T* B, int nrhs, Backend backend = Backend::Auto) {
  detail::check_dims(n, batch);
  if (batch == 0 || nrhs == 0) return;
  if (backend == Backend::Cuda) {
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_lu_solve_batched_host_f64(LU, piv, n, batch, B, nrhs));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_lu_solve_batched_host_f32(LU, piv, n, batch, B, nrhs));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  const std::int64_t nn = std::int64_t(n) * n, bn = std::int64_t(n) * nrhs;
  detail::for_batch(batch, n, [&](std::int64_t b) { detail::lu_solve(LU + b * nn, piv + b * n, n, B + b * bn, nrhs); });
}

// One-shot drivers: A is overwritten by its factor, B by the solution (batched.hpp:270-280).
template <class T>
void posv_batched(T* A, int n, std::int64_t batch, T* B, int nrhs, int* info, Backend be = Backend::Auto) {
  if (be == Backend::Cuda) {
    detail::check_dims(n, batch);
    if (batch == 0) return;
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_posv_batched_host_f64(A, n, batch, B, nrhs, info));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_posv_batched_host_f32(A, n, batch, B, nrhs, info));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  cholesky_batched<T>(A, n, batch, info, be);
  cholesky_solve_batched<T>(A, n, batch, B, nrhs, be);
}
template <class T>
void gesv_batched(T* A, int n, std::int64_t batch, T* B, int nrhs, int* piv, int* info, Backend be = Backend::Auto) {
  if (be == Backend::Cuda) {
    detail::check_dims(n, batch);
    if (!piv) throw std::invalid_argument("piv must not be null");
    if (batch == 0) return;
    if constexpr (std::is_same<T, double>::value) return detail::check_cuda(tsdx_cuda_gesv_batched_host_f64(A, n, batch, B, nrhs, piv, info));
    else if constexpr (std::is_same<T, float>::value) return detail::check_cuda(tsdx_cuda_gesv_batched_host_f32(A, n, batch, B, nrhs, piv, info));
    throw std::runtime_error("CUDA backend unavailable for this build/precision");
  }
  lu_batched<T>(A, n, batch, piv, info, be);
  lu_solve_batched<T>(A, piv, n, batch, B, nrhs, be);
}

// ------------------------------------------------- runtime-precision entry points
namespace detail {
template <class F> void with_precision(Precision p, F&& f) {
  switch (p) {
    case Precision::FP32: f(float{}); break;
    case Precision::FP64: f(double{}); break;
    case Precision::FP16: f(Half{}); break;
    case Precision::BF16: f(BFloat16{}); break;
  }
}
template <class T, class S> std::vector<T> to_t(const S* x, std::int64_t count) {
  std::vector<T> v(static_cast<std::size_t>(count));
  for (std::int64_t i = 0; i < count; ++i) v[i] = T(x[i]);
  return v;
}
template <class T> double as_d(T x) {
  if constexpr (is_native<T>::value) return static_cast<double>(x);
  else return x.v;
}
template <class T, class S> void from_t(const std::vector<T>& v, S* x) {
  for (std::size_t i = 0; i < v.size(); ++i) x[i] = static_cast<S>(as_d(v[i]));
}
}  // namespace detail

namespace detail {
// Emulated formats on the GPU (tsdx_cuda_emu_*_host, bit-identical to the CPU path):
// the reference throws here (batched.hpp:130-132); this build runs them instead.
template <class T> constexpr int emu_fmt() { return std::is_same<T, Half>::value ? 0 : 1; }
template <class S> std::vector<double> f64_copy(const S* x, std::int64_t count) {
  return std::vector<double>(x, x + count);
}
template <class S> void f64_back(const std::vector<double>& v, S* x) {
  for (std::size_t i = 0; i < v.size(); ++i) x[i] = static_cast<S>(v[i]);
}
}  // namespace detail

template <class S>
void cholesky(Precision p, S* A, int n, std::int64_t batch, int* info, Backend be = Backend::Auto) {
  detail::with_precision(p, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (std::is_same<T, S>::value) cholesky_batched<T>(A, n, batch, info, be);
    else {
      if constexpr (!is_native<T>::value) {
        if (be == Backend::Cuda) {
          detail::check_dims(n, batch);
          auto w = detail::f64_copy(A, batch * n * n);
          detail::check_cuda(tsdx_cuda_emu_factor_host(detail::emu_fmt<T>(), 0, w.data(), n, batch, nullptr, info));
          detail::f64_back(w, A);
          return;
        }
      }
      auto v = detail::to_t<T>(A, batch * n * n);
      cholesky_batched<T>(v.data(), n, batch, info, be);
      detail::from_t(v, A);
    }
  });
}
template <class S>
void lu(Precision p, S* A, int n, std::int64_t batch, int* piv, int* info, Backend be = Backend::Auto) {
  detail::with_precision(p, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (std::is_same<T, S>::value) lu_batched<T>(A, n, batch, piv, info, be);
    else {
      if constexpr (!is_native<T>::value) {
        if (be == Backend::Cuda) {
          detail::check_dims(n, batch);
          if (!piv) throw std::invalid_argument("piv must not be null");
          auto w = detail::f64_copy(A, batch * n * n);
          detail::check_cuda(tsdx_cuda_emu_factor_host(detail::emu_fmt<T>(), 1, w.data(), n, batch, piv, info));
          detail::f64_back(w, A);
          return;
        }
      }
      auto v = detail::to_t<T>(A, batch * n * n);
      lu_batched<T>(v.data(), n, batch, piv, info, be);
      detail::from_t(v, A);
    }
  });
}
template <class S>
void cholesky_solve(Precision p, const S* L, int n, std::int64_t batch, S* B, int nrhs, Backend be = Backend::Auto) {
  detail::with_precision(p, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (!is_native<T>::value) {
      if (be == Backend::Cuda) {
        detail::check_dims(n, batch);
        auto l = detail::f64_copy(L, batch * n * n);
        auto b = detail::f64_copy(B, batch * n * nrhs);
        detail::check_cuda(tsdx_cuda_emu_solve_host(detail::emu_fmt<T>(), 0, l.data(), nullptr, n, batch, b.data(), nrhs));
        detail::f64_back(b, B);
        return;
      }
    }
    auto l = detail::to_t<T>(L, batch * n * n);
    auto b = detail::to_t<T>(B, batch * n * nrhs);
    cholesky_solve_batched<T>(l.data(), n, batch, b.data(), nrhs, be);
    detail::from_t(b, B);
  });
}
template <class S>
void lu_solve(Precision p, const S* LU, const int* piv, int n, std::int64_t batch, S* B, int nrhs, Backend be = Backend::Auto) {
  detail::with_precision(p, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (!is_native<T>::value) {
      if (be == Backend::Cuda) {
        detail::check_dims(n, batch);
        auto l = detail::f64_copy(LU, batch * n * n);
        auto b = detail::f64_copy(B, batch * n * nrhs);
        detail::check_cuda(tsdx_cuda_emu_solve_host(detail::emu_fmt<T>(), 1, l.data(), piv, n, batch, b.data(), nrhs));
        detail::f64_back(b, B);
        return;
      }
    }
    auto l = detail::to_t<T>(LU, batch * n * n);
    auto b = detail::to_t<T>(B, batch * n * nrhs);
    lu_solve_batched<T>(l.data(), piv, n, batch, b.data(), nrhs, be);
    detail::from_t(b, B);
  });
}
template <class S>
void round_to(Precision p, S* x, std::int64_t count) {
  if (p == Precision::FP64) return;
  for (std::int64_t i = 0; i < count; ++i) {
    const float f = static_cast<float>(x[i]);
    x[i] = static_cast<S>(p == Precision::FP32 ? f : p == Precision::FP16 ? detail::round_fp16(f) : detail::round_bf16(f));
  }
}

// ------------------------------------------ long-double ground truth & metrics
namespace detail {
using LD = long double;
inline void ld_solve(const double* A, const double* b, int n, LD* x) {
  std::vector<LD> a(static_cast<std::size_t>(n) * n);
  for (int i = 0; i < n * n; ++i) a[i] = A[i];
  for (int i = 0; i < n; ++i) x[i] = b[i];
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i) if (std::fabs(a[i * n + k]) > std::fabs(a[p * n + k])) p = i;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
      std::swap(x[k], x[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const LD f = a[i * n + k] / a[k * n + k];
      for (int j = k + 1; j < n; ++j) a[i * n + j] -= f * a[k * n + j];
      x[i] -= f * x[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    LD s = x[i];
    for (int j = i + 1; j < n; ++j) s -= a[i * n + j] * x[j];
    x[i] = s / a[i * n + i];
  }
}
inline LD fro(const double* a, int cnt) { LD s = 0; for (int i = 0; i < cnt; ++i) s += (LD)a[i] * a[i]; return std::sqrt(s); }
}  // namespace detail

inline void chol_backward_error(const double* A, const double* L, int n, std::int64_t batch, double* out) {
  parallel_for(batch, [&](std::int64_t b) {
    const double* a = A + b * n * n; const double* l = L + b * n * n;
    detail::LD num = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        detail::LD s = 0;
        for (int k = 0; k <= std::min(i, j); ++k) s += (detail::LD)l[i * n + k] * l[j * n + k];
        const detail::LD d = (detail::LD)a[i * n + j] - s;
        num += d * d;
      }
    out[b] = static_cast<double>(std::sqrt(num) / detail::fro(a, n * n));
  });
}
inline void lu_backward_error(const double* A, const double* LU, const int* piv, int n, std::int64_t batch, double* out) {
  parallel_for(batch, [&](std::int64_t b) {
    const double* a = A + b * n * n; const double* f = LU + b * n * n; const int* pv = piv + b * n;
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) std::swap(perm[k], perm[pv[k]]);
    detail::LD num = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        detail::LD s = 0;
        for (int k = 0; k <= std::min(i, j); ++k) s += ((k == i) ? (detail::LD)1 : (detail::LD)f[i * n + k]) * f[k * n + j];
        const detail::LD d = (detail::LD)a[perm[i] * n + j] - s;
        num += d * d;
      }
    out[b] = static_cast<double>(std::sqrt(num) / detail::fro(a, n * n));
  });
}
inline void solve_backward_error(const double* A, const double* x, const double* bb, int n, std::int64_t batch, double* out) {
  parallel_for(batch, [&](std::int64_t b) {
    const double* a = A + b * n * n; const double* xv = x + b * n; const double* rhs = bb + b * n;
    detail::LD num = 0;
    for (int i = 0; i < n; ++i) {
      detail::LD s = rhs[i];
      for (int j = 0; j < n; ++j) s -= (detail::LD)a[i * n + j] * xv[j];
      num += s * s;
    }
    out[b] = static_cast<double>(std::sqrt(num) / (detail::fro(a, n * n) * detail::fro(xv, n) + detail::fro(rhs, n)));
  });
}
inline void reference_solve(const double* A, const double* b, int n, std::int64_t batch, double* x) {
  parallel_for(batch, [&](std::int64_t m) {
    std::vector<detail::LD> xr(n);
    detail::ld_solve(A + m * n * n, b + m * n, n, xr.data());
    for (int i = 0; i < n; ++i) x[m * n + i] = static_cast<double>(xr[i]);
  });
}
inline void solve_forward_error(const double* A, const double* x, const double* b, int n, std::int64_t batch, double* out) {
  parallel_for(batch, [&](std::int64_t m) {
    std::vector<detail::LD> xr(n);
    detail::ld_solve(A + m * n * n, b + m * n, n, xr.data());
    detail::LD num = 0, den = 0;
    for (int i = 0; i < n; ++i) { const detail::LD d = (detail::LD)x[m * n + i] - xr[i]; num += d * d; den += xr[i] * xr[i]; }
    out[m] = static_cast<double>(std::sqrt(num / den));
  });
}

}  // namespace tsdx
