/*
 * CPU oracle for the batched small-matrix solver: a plain-C restatement of the
 * reference's per-matrix arithmetic (TinySolverDx include/tinysolverdx/kernels.hpp,
 * precision.hpp) and of its long-double ground truth and error metrics
 * (src/runtime.cpp:162-260).
 *
 * THIS IS TEST INFRASTRUCTURE. Only the test-suite, the smoke check and the
 * CPU-baseline leg of the benchmark load it, and only as the checker. The GPU
 * product path never calls into this file.
 *
 * Parity pin: tests/test_oracle.py compares every routine here bit-for-bit
 * against the reference library compiled from its own sources
 * (oracle/_ref/libtsdx_ref.so, built by oracle/Makefile) and against the
 * committed golden vectors in tests/golden/.
 *
 * Floating-point contract. The reference is built with -O3 -march=native and
 * GCC's default -ffp-contract=fast, so every `x -= a * b` in kernels.hpp becomes
 * one fused multiply-add. This file spells those contractions out as fma()
 * and is compiled with -ffp-contract=off so that no other contraction happens.
 * Divisions and square roots are IEEE (correctly rounded) as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* Per-matrix kernels, generated for float (suffix f) and double (suffix d).  */
/* ------------------------------------------------------------------------- */
#define ORC_KERNELS(T, S, FMA, SQRT, FABS)                                         \
  /* kernels.hpp:18-37  left-looking row Cholesky; early return on failure.    */  \
  /* GCC vectorises the dot product s -= ai[k]*aj[k] in 16-byte groups with an  */  \
  /* in-order reduction: each complete group of G = 16/sizeof(T) terms is a     */  \
  /* separately rounded product then subtraction, the remaining j mod G terms   */  \
  /* are contracted to FMA (pinned against the compiled reference). The double */  \
  /* n = 3 instantiation is not vectorised: all its terms are fused.            */  \
  ORC_API int orc_cholesky_rm_##S(T* a, int n) {                                   \
    const int G = (sizeof(T) == 8 && n == 3) ? 64 : 16 / (int)sizeof(T);           \
    for (int i = 0; i < n; ++i) {                                                  \
      T* ai = a + (int64_t)i * n;                                                  \
      for (int j = 0; j <= i; ++j) {                                               \
        const T* aj = a + (int64_t)j * n;                                          \
        T s = ai[j];                                                               \
        const int kv = j / G * G;                                                  \
        for (int k = 0; k < kv; ++k) s = s - ai[k] * aj[k];                        \
        for (int k = kv; k < j; ++k) s = FMA(-ai[k], aj[k], s);                    \
        if (j == i) {                                                              \
          if (!(s > (T)0)) return i + 1;                                           \
          ai[i] = SQRT(s);                                                         \
        } else {                                                                   \
          ai[j] = s / aj[j];                                                       \
        }                                                                          \
      }                                                                            \
    }                                                                              \
    for (int i = 0; i < n; ++i)                                                    \
      for (int j = i + 1; j < n; ++j) a[(int64_t)i * n + j] = (T)0;                \
    return 0;                                                                      \
  }                                                                                \
  /* kernels.hpp:41-54  right-looking column Cholesky ("naive" backend). */        \
  ORC_API int orc_cholesky_naive_##S(T* a, int n) {                                \
    for (int j = 0; j < n; ++j) {                                                  \
      for (int k = 0; k < j; ++k)                                                  \
        for (int i = j; i < n; ++i)                                                \
          a[i * n + j] = FMA(-a[i * n + k], a[j * n + k], a[i * n + j]);           \
      if (!(a[j * n + j] > (T)0)) return j + 1;                                    \
      const T d = SQRT(a[j * n + j]);                                              \
      a[j * n + j] = d;                                                            \
      for (int i = j + 1; i < n; ++i) a[i * n + j] /= d;                           \
    }                                                                              \
    for (int i = 0; i < n; ++i)                                                    \
      for (int j = i + 1; j < n; ++j) a[i * n + j] = (T)0;                         \
    return 0;                                                                      \
  }                                                                                \
  /* kernels.hpp:57-87 restated for one lane: a non-positive pivot records      */ \
  /* info once, is replaced by 1 and the factorization continues; the upper     */ \
  /* triangle is always zeroed ("simd" backend semantics). The compile-time-N   */ \
  /* instantiations (n <= 16, batched.hpp:88-91) contract s -= x*y to one FMA;  */ \
  /* the runtime-N one (n >= 17, chol_tile_rt, batched.hpp:85) rounds the       */ \
  /* product and the subtraction separately (pinned against the compiled       */ \
  /* reference).                                                                */ \
  ORC_API int orc_cholesky_tile_##S(T* a, int n) {                                 \
    int info = 0;                                                                  \
    const int fused = n <= 16;                                                     \
    for (int i = 0; i < n; ++i) {                                                  \
      for (int j = 0; j <= i; ++j) {                                               \
        T s = a[i * n + j];                                                        \
        if (fused)                                                                 \
          for (int k = 0; k < j; ++k) s = FMA(-a[i * n + k], a[j * n + k], s);     \
        else                                                                       \
          for (int k = 0; k < j; ++k) s = s - a[i * n + k] * a[j * n + k];         \
        if (j == i) {                                                              \
          const int bad = !(s > (T)0);                                             \
          if (bad && info == 0) info = i + 1;                                      \
          s = bad ? (T)1 : s;                                                      \
          s = SQRT(s);                                                             \
        } else {                                                                   \
          s /= a[j * n + j];                                                       \
        }                                                                          \
        a[i * n + j] = s;                                                          \
      }                                                                            \
    }                                                                              \
    for (int i = 0; i < n; ++i)                                                    \
      for (int j = i + 1; j < n; ++j) a[i * n + j] = (T)0;                         \
    return info;                                                                   \
  }                                                                                \
  /* kernels.hpp:91-119  right-looking GEPP, strict '>' argmax (first maximum  */  \
  /* wins, NaN never wins), full-row swap, a zero pivot records info and skips */  \
  /* the elimination of that column.                                           */  \
  ORC_API int orc_lu_rm_##S(T* a, int n, int* piv) {                               \
    int info = 0;                                                                  \
    for (int k = 0; k < n; ++k) {                                                  \
      int p = k;                                                                   \
      T best = FABS(a[k * n + k]);                                                 \
      for (int i = k + 1; i < n; ++i) {                                            \
        const T v = FABS(a[i * n + k]);                                            \
        if (v > best) { best = v; p = i; }                                         \
      }                                                                            \
      piv[k] = p;                                                                  \
      if (p != k)                                                                  \
        for (int j = 0; j < n; ++j) {                                              \
          const T t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; \
        }                                                                          \
      const T pk = a[k * n + k];                                                   \
      if (pk == (T)0) { if (info == 0) info = k + 1; continue; }                   \
      const T* rk = a + k * n;                                                     \
      for (int i = k + 1; i < n; ++i) {                                            \
        T* ri = a + i * n;                                                         \
        const T f = ri[k] / pk;                                                    \
        ri[k] = f;                                                                 \
        for (int j = k + 1; j < n; ++j) ri[j] = FMA(-f, rk[j], ri[j]);             \
      }                                                                            \
    }                                                                              \
    return info;                                                                   \
  }                                                                                \
  /* kernels.hpp:121-138  textbook column-oriented GEPP ("naive" backend). */      \
  ORC_API int orc_lu_naive_##S(T* a, int n, int* piv) {                            \
    int info = 0;                                                                  \
    for (int k = 0; k < n; ++k) {                                                  \
      int p = k;                                                                   \
      for (int i = k + 1; i < n; ++i)                                              \
        if (FABS(a[i * n + k]) > FABS(a[p * n + k])) p = i;                        \
      piv[k] = p;                                                                  \
      if (p != k)                                                                  \
        for (int j = 0; j < n; ++j) {                                              \
          T t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t;       \
        }                                                                          \
      if (a[k * n + k] == (T)0) { if (info == 0) info = k + 1; continue; }         \
      for (int j = k + 1; j < n; ++j)                                              \
        for (int i = k + 1; i < n; ++i)                                            \
          a[i * n + j] = FMA(-(a[i * n + k] / a[k * n + k]), a[k * n + j],         \
                             a[i * n + j]);                                        \
      for (int i = k + 1; i < n; ++i) a[i * n + k] /= a[k * n + k];                \
    }                                                                              \
    return info;                                                                   \
  }                                                                                \
  /* kernels.hpp:141-180 restated for one lane: a zero pivot records info and  */  \
  /* is replaced by 1 for the scaling; elimination still runs ("simd").        */  \
  ORC_API int orc_lu_tile_##S(T* a, int n, int* piv) {                             \
    int info = 0;                                                                  \
    for (int k = 0; k < n; ++k) {                                                  \
      int p = k;                                                                   \
      T best = FABS(a[k * n + k]);                                                 \
      for (int i = k + 1; i < n; ++i) {                                            \
        const T v = FABS(a[i * n + k]);                                            \
        const int gt = v > best;                                                   \
        best = gt ? v : best;                                                      \
        p = gt ? i : p;                                                            \
      }                                                                            \
      piv[k] = p;                                                                  \
      if (p != k)                                                                  \
        for (int j = 0; j < n; ++j) {                                              \
          const T t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; \
        }                                                                          \
      const T pk = a[k * n + k];                                                   \
      const int zero = (pk == (T)0);                                               \
      if (zero && info == 0) info = k + 1;                                         \
      const T d = zero ? (T)1 : pk;                                                \
      const T* rk = a + k * n;                                                     \
      for (int i = k + 1; i < n; ++i) {                                            \
        T* ri = a + i * n;                                                         \
        const T f = ri[k] / d;                                                     \
        ri[k] = f;                                                                 \
        for (int j = k + 1; j < n; ++j) ri[j] = FMA(-f, rk[j], ri[j]);             \
      }                                                                            \
    }                                                                              \
    return info;                                                                   \
  }                                                                                \
  /* kernels.hpp:184-202  forward then backward substitution with L (lower). */    \
  ORC_API void orc_cholesky_solve_rm_##S(const T* L, int n, T* B, int nrhs) {      \
    for (int i = 0; i < n; ++i) {                                                  \
      for (int k = 0; k < i; ++k) {                                                \
        const T lik = L[i * n + k];                                                \
        for (int r = 0; r < nrhs; ++r)                                             \
          B[i * nrhs + r] = FMA(-lik, B[k * nrhs + r], B[i * nrhs + r]);           \
      }                                                                            \
      const T d = L[i * n + i];                                                    \
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] /= d;                         \
    }                                                                              \
    for (int i = n - 1; i >= 0; --i) {                                             \
      for (int k = i + 1; k < n; ++k) {                                            \
        const T lki = L[k * n + i];                                                \
        for (int r = 0; r < nrhs; ++r)                                             \
          B[i * nrhs + r] = FMA(-lki, B[k * nrhs + r], B[i * nrhs + r]);           \
      }                                                                            \
      const T d = L[i * n + i];                                                    \
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] /= d;                         \
    }                                                                              \
  }                                                                                \
  /* kernels.hpp:204-227  pivots applied in k order, unit-L forward, U back. */    \
  ORC_API void orc_lu_solve_rm_##S(const T* LU, const int* piv, int n, T* B,       \
                                   int nrhs) {                                     \
    for (int k = 0; k < n; ++k)                                                    \
      if (piv[k] != k)                                                             \
        for (int r = 0; r < nrhs; ++r) {                                           \
          const T t = B[k * nrhs + r];                                             \
          B[k * nrhs + r] = B[piv[k] * nrhs + r];                                  \
          B[piv[k] * nrhs + r] = t;                                                \
        }                                                                          \
    for (int i = 0; i < n; ++i)                                                    \
      for (int k = 0; k < i; ++k) {                                                \
        const T lik = LU[i * n + k];                                               \
        for (int r = 0; r < nrhs; ++r)                                             \
          B[i * nrhs + r] = FMA(-lik, B[k * nrhs + r], B[i * nrhs + r]);           \
      }                                                                            \
    for (int i = n - 1; i >= 0; --i) {                                             \
      for (int k = i + 1; k < n; ++k) {                                            \
        const T uik = LU[i * n + k];                                               \
        for (int r = 0; r < nrhs; ++r)                                             \
          B[i * nrhs + r] = FMA(-uik, B[k * nrhs + r], B[i * nrhs + r]);           \
      }                                                                            \
      const T d = LU[i * n + i];                                                   \
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] /= d;                         \
    }                                                                              \
  }

ORC_KERNELS(double, d, fma, sqrt, fabs)
ORC_KERNELS(float, f, fmaf, sqrtf, fabsf)

/* ------------------------------------------------------------------------- */
/* Batch drivers. The reference's chunking and lane interleaving never change */
/* a result (lanes are independent; batched.hpp:153-178, :217-243), so the    */
/* oracle simply loops. backend: 1 naive, 2 scalar, 3 simd.                   */
/* batched.hpp:187: the reference's Auto picks scalar LU for n >= 25, else    */
/* simd; Auto Cholesky is simd for float/double (batched.hpp:46-50).          */
/* ------------------------------------------------------------------------- */
enum { ORC_AUTO = 0, ORC_NAIVE = 1, ORC_SCALAR = 2, ORC_SIMD = 3 };

#define ORC_DRIVERS(T, S)                                                          \
  ORC_API void orc_cholesky_batched_##S(T* A, int n, int64_t batch, int* info,     \
                                        int backend) {                             \
    const int64_t nn = (int64_t)n * n;                                             \
    if (backend == ORC_AUTO) backend = ORC_SIMD;                                   \
    for (int64_t b = 0; b < batch; ++b) {                                          \
      int r;                                                                       \
      if (backend == ORC_NAIVE) r = orc_cholesky_naive_##S(A + b * nn, n);         \
      else if (backend == ORC_SCALAR) r = orc_cholesky_rm_##S(A + b * nn, n);      \
      else r = orc_cholesky_tile_##S(A + b * nn, n);                               \
      if (info) info[b] = r;                                                       \
    }                                                                              \
  }                                                                                \
  ORC_API void orc_lu_batched_##S(T* A, int n, int64_t batch, int* piv, int* info, \
                                  int backend) {                                   \
    const int64_t nn = (int64_t)n * n;                                             \
    if (backend == ORC_AUTO) backend = n >= 25 ? ORC_SCALAR : ORC_SIMD;            \
    for (int64_t b = 0; b < batch; ++b) {                                          \
      int r;                                                                       \
      if (backend == ORC_NAIVE) r = orc_lu_naive_##S(A + b * nn, n, piv + b * n);  \
      else if (backend == ORC_SCALAR) r = orc_lu_rm_##S(A + b * nn, n, piv + b * n);\
      else r = orc_lu_tile_##S(A + b * nn, n, piv + b * n);                        \
      if (info) info[b] = r;                                                       \
    }                                                                              \
  }                                                                                \
  ORC_API void orc_cholesky_solve_batched_##S(const T* L, int n, int64_t batch,    \
                                              T* B, int nrhs) {                    \
    const int64_t nn = (int64_t)n * n, bn = (int64_t)n * nrhs;                     \
    for (int64_t b = 0; b < batch; ++b)                                            \
      orc_cholesky_solve_rm_##S(L + b * nn, n, B + b * bn, nrhs);                  \
  }                                                                                \
  ORC_API void orc_lu_solve_batched_##S(const T* LU, const int* piv, int n,        \
                                        int64_t batch, T* B, int nrhs) {           \
    const int64_t nn = (int64_t)n * n, bn = (int64_t)n * nrhs;                     \
    for (int64_t b = 0; b < batch; ++b)                                            \
      orc_lu_solve_rm_##S(LU + b * nn, piv + b * n, n, B + b * bn, nrhs);          \
  }

ORC_DRIVERS(double, d)
ORC_DRIVERS(float, f)

/* ------------------------------------------------------------------------- */
/* fp16 / bf16 rounding and per-operation-rounding emulation                  */
/* (precision.hpp:41-97). Every +,-,*,/ and sqrt is computed in float and      */
/* rounded to the target format, with no wide accumulator.                     */
/* ------------------------------------------------------------------------- */
static uint32_t f2u(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static float u2f(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* precision.hpp:41-55  RNE to binary16, subnormal quantum 2^-24, overflow to inf. */
ORC_API float orc_round_fp16(float x) {
  const uint32_t u = f2u(x), sign = u & 0x80000000u, a = u & 0x7fffffffu;
  if (a >= 0x7f800000u) return x;
  const float ax = u2f(a);
  if (ax >= 65520.0f) return u2f(sign | 0x7f800000u);
  if (ax < 6.103515625e-05f) {
    const float q = 5.9604644775390625e-08f;
    return u2f(sign | f2u(nearbyintf(ax / q) * q));
  }
  uint32_t r = a + 0xfffu + ((a >> 13) & 1u);
  r &= ~0x1fffu;
  return u2f(sign | r);
}
/* precision.hpp:58-65  RNE to bfloat16; NaN passes through. */
ORC_API float orc_round_bf16(float x) {
  const uint32_t u = f2u(x), a = u & 0x7fffffffu;
  if (a > 0x7f800000u) return x;
  uint32_t r = a + 0x7fffu + ((a >> 16) & 1u);
  r &= ~0xffffu;
  return u2f((u & 0x80000000u) | r);
}

typedef float (*orc_rnd)(float);
static orc_rnd rounder(int fmt) { return fmt == 0 ? orc_round_fp16 : orc_round_bf16; }

/* cholesky_rm over Emu<F> (kernels.hpp:18-37 with precision.hpp:84-97). */
static int emu_cholesky_rm(float* a, int n, orc_rnd R) {
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j <= i; ++j) {
      float s = a[i * n + j];
      for (int k = 0; k < j; ++k) s = R(s - R(a[i * n + k] * a[j * n + k]));
      if (j == i) {
        if (!(s > 0.0f)) return i + 1;
        a[i * n + i] = R(sqrtf(s));
      } else {
        a[i * n + j] = R(s / a[j * n + j]);
      }
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) a[i * n + j] = 0.0f;
  return 0;
}
/* lu_rm over Emu<F>. t_abs(x) is x < 0 ? -x : x (precision.hpp:103). */
static int emu_lu_rm(float* a, int n, int* piv, orc_rnd R) {
  int info = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    float best = a[k * n + k] < 0.0f ? -a[k * n + k] : a[k * n + k];
    for (int i = k + 1; i < n; ++i) {
      const float v = a[i * n + k] < 0.0f ? -a[i * n + k] : a[i * n + k];
      if (v > best) { best = v; p = i; }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) { float t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; }
    const float pk = a[k * n + k];
    if (pk == 0.0f) { if (info == 0) info = k + 1; continue; }
    for (int i = k + 1; i < n; ++i) {
      const float f = R(a[i * n + k] / pk);
      a[i * n + k] = f;
      for (int j = k + 1; j < n; ++j) a[i * n + j] = R(a[i * n + j] - R(f * a[k * n + j]));
    }
  }
  return info;
}
static void emu_cholesky_solve_rm(const float* L, int n, float* B, int nrhs, orc_rnd R) {
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k)
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] - R(L[i * n + k] * B[k * nrhs + r]));
    for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] / L[i * n + i]);
  }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k)
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] - R(L[k * n + i] * B[k * nrhs + r]));
    for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] / L[i * n + i]);
  }
}
static void emu_lu_solve_rm(const float* LU, const int* piv, int n, float* B, int nrhs, orc_rnd R) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k)
      for (int r = 0; r < nrhs; ++r) { float t = B[k * nrhs + r]; B[k * nrhs + r] = B[piv[k] * nrhs + r]; B[piv[k] * nrhs + r] = t; }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < i; ++k)
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] - R(LU[i * n + k] * B[k * nrhs + r]));
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k)
      for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] - R(LU[i * n + k] * B[k * nrhs + r]));
    for (int r = 0; r < nrhs; ++r) B[i * nrhs + r] = R(B[i * nrhs + r] / LU[i * n + i]);
  }
}

/* Runtime-precision entry points for the emulated formats over double storage
 * (runtime.cpp:81-91 to_t/from_t: Emu(double x) rounds x to float first, then
 * to the format). fmt: 0 fp16, 1 bf16. The reference resolves emulated types to
 * the scalar backend (batched.hpp:46-50). */
ORC_API void orc_emu_cholesky(int fmt, double* A, int n, int64_t batch, int* info) {
  orc_rnd R = rounder(fmt);
  const int64_t nn = (int64_t)n * n;
  float* w = (float*)malloc(sizeof(float) * (size_t)nn);
  for (int64_t b = 0; b < batch; ++b) {
    for (int64_t e = 0; e < nn; ++e) w[e] = R((float)A[b * nn + e]);
    const int r = emu_cholesky_rm(w, n, R);
    if (info) info[b] = r;
    for (int64_t e = 0; e < nn; ++e) A[b * nn + e] = (double)w[e];
  }
  free(w);
}
ORC_API void orc_emu_lu(int fmt, double* A, int n, int64_t batch, int* piv, int* info) {
  orc_rnd R = rounder(fmt);
  const int64_t nn = (int64_t)n * n;
  float* w = (float*)malloc(sizeof(float) * (size_t)nn);
  for (int64_t b = 0; b < batch; ++b) {
    for (int64_t e = 0; e < nn; ++e) w[e] = R((float)A[b * nn + e]);
    const int r = emu_lu_rm(w, n, piv + b * n, R);
    if (info) info[b] = r;
    for (int64_t e = 0; e < nn; ++e) A[b * nn + e] = (double)w[e];
  }
  free(w);
}
ORC_API void orc_emu_cholesky_solve(int fmt, const double* L, int n, int64_t batch, double* B, int nrhs) {
  orc_rnd R = rounder(fmt);
  const int64_t nn = (int64_t)n * n, bn = (int64_t)n * nrhs;
  float* l = (float*)malloc(sizeof(float) * (size_t)nn);
  float* x = (float*)malloc(sizeof(float) * (size_t)bn);
  for (int64_t b = 0; b < batch; ++b) {
    for (int64_t e = 0; e < nn; ++e) l[e] = R((float)L[b * nn + e]);
    for (int64_t e = 0; e < bn; ++e) x[e] = R((float)B[b * bn + e]);
    emu_cholesky_solve_rm(l, n, x, nrhs, R);
    for (int64_t e = 0; e < bn; ++e) B[b * bn + e] = (double)x[e];
  }
  free(l); free(x);
}
ORC_API void orc_emu_lu_solve(int fmt, const double* LU, const int* piv, int n, int64_t batch, double* B, int nrhs) {
  orc_rnd R = rounder(fmt);
  const int64_t nn = (int64_t)n * n, bn = (int64_t)n * nrhs;
  float* l = (float*)malloc(sizeof(float) * (size_t)nn);
  float* x = (float*)malloc(sizeof(float) * (size_t)bn);
  for (int64_t b = 0; b < batch; ++b) {
    for (int64_t e = 0; e < nn; ++e) l[e] = R((float)LU[b * nn + e]);
    for (int64_t e = 0; e < bn; ++e) x[e] = R((float)B[b * bn + e]);
    emu_lu_solve_rm(l, piv + b * n, n, x, nrhs, R);
    for (int64_t e = 0; e < bn; ++e) B[b * bn + e] = (double)x[e];
  }
  free(l); free(x);
}
/* runtime.cpp:143-150  round_to over double storage. prec: 0 fp32, 1 fp64, 2 fp16, 3 bf16. */
ORC_API void orc_round_to(int prec, double* x, int64_t count) {
  if (prec == 1) return;
  for (int64_t i = 0; i < count; ++i) {
    const float f = (float)x[i];
    x[i] = (double)(prec == 0 ? f : prec == 2 ? orc_round_fp16(f) : orc_round_bf16(f));
  }
}

/* ------------------------------------------------------------------------- */
/* Long-double ground truth and error metrics (runtime.cpp:162-260).         */
/* On x86-64 long double is the 80-bit x87 format (64-bit mantissa).         */
/* ------------------------------------------------------------------------- */
typedef long double LD;

/* runtime.cpp:167-189  GEPP solve in long double on a copy. */
static void ld_solve(const double* A, const double* b, int n, LD* x, LD* a) {
  for (int i = 0; i < n * n; ++i) a[i] = A[i];
  for (int i = 0; i < n; ++i) x[i] = b[i];
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i) if (fabsl(a[i * n + k]) > fabsl(a[p * n + k])) p = i;
    if (p != k) {
      for (int j = 0; j < n; ++j) { LD t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; }
      LD t = x[k]; x[k] = x[p]; x[p] = t;
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
static LD fro(const double* a, int cnt) { LD s = 0; for (int i = 0; i < cnt; ++i) s += (LD)a[i] * a[i]; return sqrtl(s); }

/* runtime.cpp:194-207  ||A - L L^T||_F / ||A||_F */
ORC_API void orc_chol_backward_error(const double* A, const double* L, int n, int64_t batch, double* out) {
  for (int64_t b = 0; b < batch; ++b) {
    const double* a = A + b * n * n; const double* l = L + b * n * n;
    LD num = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        LD s = 0;
        const int m = i < j ? i : j;
        for (int k = 0; k <= m; ++k) s += (LD)l[i * n + k] * l[j * n + k];
        const LD d = (LD)a[i * n + j] - s;
        num += d * d;
      }
    out[b] = (double)(sqrtl(num) / fro(a, n * n));
  }
}
/* runtime.cpp:209-228  ||P A - L U||_F / ||A||_F with the pivots applied in order. */
ORC_API void orc_lu_backward_error(const double* A, const double* LU, const int* piv, int n, int64_t batch, double* out) {
  int perm[64];
  for (int64_t b = 0; b < batch; ++b) {
    const double* a = A + b * n * n; const double* f = LU + b * n * n; const int* pv = piv + b * n;
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) { int t = perm[k]; perm[k] = perm[pv[k]]; perm[pv[k]] = t; }
    LD num = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        LD s = 0;
        const int m = i < j ? i : j;
        for (int k = 0; k <= m; ++k) {
          const LD lik = (k == i) ? (LD)1 : (LD)f[i * n + k];
          s += lik * f[k * n + j];
        }
        const LD d = (LD)a[perm[i] * n + j] - s;
        num += d * d;
      }
    out[b] = (double)(sqrtl(num) / fro(a, n * n));
  }
}
/* runtime.cpp:230-242  ||b - A x||_2 / (||A||_F ||x||_2 + ||b||_2) */
ORC_API void orc_solve_backward_error(const double* A, const double* x, const double* bb, int n, int64_t batch, double* out) {
  for (int64_t b = 0; b < batch; ++b) {
    const double* a = A + b * n * n; const double* xv = x + b * n; const double* rhs = bb + b * n;
    LD num = 0;
    for (int i = 0; i < n; ++i) {
      LD s = rhs[i];
      for (int j = 0; j < n; ++j) s -= (LD)a[i * n + j] * xv[j];
      num += s * s;
    }
    const LD den = fro(a, n * n) * fro(xv, n) + fro(rhs, n);
    out[b] = (double)(sqrtl(num) / den);
  }
}
/* runtime.cpp:244-250 */
ORC_API void orc_reference_solve(const double* A, const double* b, int n, int64_t batch, double* x) {
  LD xr[64], a[64 * 64];
  for (int64_t m = 0; m < batch; ++m) {
    ld_solve(A + m * n * n, b + m * n, n, xr, a);
    for (int i = 0; i < n; ++i) x[m * n + i] = (double)xr[i];
  }
}
/* runtime.cpp:252-260  ||x - x_ref||_2 / ||x_ref||_2 */
ORC_API void orc_solve_forward_error(const double* A, const double* x, const double* b, int n, int64_t batch, double* out) {
  LD xr[64], a[64 * 64];
  for (int64_t m = 0; m < batch; ++m) {
    ld_solve(A + m * n * n, b + m * n, n, xr, a);
    LD num = 0, den = 0;
    for (int i = 0; i < n; ++i) { const LD d = (LD)x[m * n + i] - xr[i]; num += d * d; den += xr[i] * xr[i]; }
    out[m] = (double)sqrtl(num / den);
  }
}
