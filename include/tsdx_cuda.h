/*
 * tsdx_cuda.h — C-ABI of the B200 (sm_100a) batched small-matrix solver.
 *
 * This is the drop-in boundary behind TinySolverDx's batched API. Every entry
 * point takes plain pointers and sizes and returns an int status (0 = success,
 * negative = error, see TSDX_ERR_*); numerical failure is never an error but a
 * LAPACK-style info code, exactly as in the reference.
 *
 * Layouts (TinySolverDx include/tinysolverdx/batched.hpp:1-6, :247):
 *   A    (batch, n, n)   row-major, matrices contiguous; overwritten by the factor
 *   B    (batch, n, nrhs) row-major; overwritten by the solution
 *   piv  (batch, n) int32, 0-based LAPACK sequential pivots (piv[k] = row swapped with k)
 *   info (batch) int32 or NULL: 0 ok, k > 0 first failing pivot (1-based)
 * Sizes: 1 <= n <= 64, batch >= 0, nrhs >= 0.
 *
 * Two families:
 *  - tsdx_cuda_*      : DEVICE pointers, asynchronous on `stream` (a cudaStream_t
 *                       passed as void*, NULL = the legacy default stream).
 *  - tsdx_cuda_*_host : HOST pointers, synchronous, same semantics as the
 *                       reference's CUDA backend (copy in, compute, copy out).
 *
 * Numerical contract: Cholesky factors, LU factors, pivots and info are
 * bit-identical to the reference CPU library's default backends (Cholesky:
 * kernels.hpp:57-87 as the simd backend compiles it; LU: kernels.hpp:91-119);
 * solutions agree to rounding (column-oriented back substitution).
 */
#ifndef TSDX_CUDA_H
#define TSDX_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSDX_OK 0
#define TSDX_ERR_N (-1)     /* n outside [1, 64] (batched.hpp:39-41)              */
#define TSDX_ERR_BATCH (-2) /* batch < 0 (batched.hpp:42)                          */
#define TSDX_ERR_NULL (-3)  /* a required pointer is NULL (batched.hpp:184 for piv) */
#define TSDX_ERR_NRHS (-4)  /* nrhs < 0                                            */
#define TSDX_ERR_CUDA (-5)  /* a CUDA runtime call failed; see tsdx_cuda_last_error */
#define TSDX_ERR_NODEV (-6) /* no CUDA device is visible                           */
#define TSDX_ERR_TOO_LARGE (-7) /* count above a fixed capacity; see tsdx_cuda_last_error */

/* 1 if a CUDA device is visible (replaces tsdx::cuda::available, cuda_backend.hpp:9). */
int tsdx_cuda_available(void);
/* Message of the last TSDX_ERR_CUDA on the calling thread ("" if none). */
const char* tsdx_cuda_last_error(void);
/* Kernels of this library launched since load (all threads); for accounting. */
int64_t tsdx_cuda_launch_count(void);

/* ---- device-pointer, stream-ordered API ---------------------------------------
 * potrf  replaces cholesky_batched<T>(A, n, batch, info, Backend::Cuda)  batched.hpp:121-133
 * getrf  replaces lu_batched<T>(A, n, batch, piv, info, Backend::Cuda)    batched.hpp:181-197
 * potrs  replaces cholesky_solve_batched<T>(L, n, batch, B, nrhs)         batched.hpp:248-257
 * getrs  replaces lu_solve_batched<T>(LU, piv, n, batch, B, nrhs)         batched.hpp:259-268
 * posv   replaces posv_batched<T>(A, n, batch, B, nrhs, info, be)         batched.hpp:271-275
 * gesv   replaces gesv_batched<T>(A, n, batch, B, nrhs, piv, info, be)    batched.hpp:276-280
 */
int tsdx_cuda_potrf_f32(float* A, int n, int64_t batch, int* info, void* stream);
int tsdx_cuda_potrf_f64(double* A, int n, int64_t batch, int* info, void* stream);
int tsdx_cuda_getrf_f32(float* A, int n, int64_t batch, int* piv, int* info, void* stream);
int tsdx_cuda_getrf_f64(double* A, int n, int64_t batch, int* piv, int* info, void* stream);
int tsdx_cuda_potrs_f32(const float* L, int n, int64_t batch, float* B, int nrhs, void* stream);
int tsdx_cuda_potrs_f64(const double* L, int n, int64_t batch, double* B, int nrhs, void* stream);
int tsdx_cuda_getrs_f32(const float* LU, const int* piv, int n, int64_t batch, float* B, int nrhs, void* stream);
int tsdx_cuda_getrs_f64(const double* LU, const int* piv, int n, int64_t batch, double* B, int nrhs, void* stream);
int tsdx_cuda_posv_f32(float* A, int n, int64_t batch, float* B, int nrhs, int* info, void* stream);
int tsdx_cuda_posv_f64(double* A, int n, int64_t batch, double* B, int nrhs, int* info, void* stream);
int tsdx_cuda_gesv_f32(float* A, int n, int64_t batch, float* B, int nrhs, int* piv, int* info, void* stream);
int tsdx_cuda_gesv_f64(double* A, int n, int64_t batch, double* B, int nrhs, int* piv, int* info, void* stream);

/* ---- host-pointer, synchronous API ---------------------------------------------
 * cholesky_batched_host / lu_batched_host replace tsdx::cuda::cholesky_batched /
 * tsdx::cuda::lu_batched (cuda_backend.hpp:10-11, cuda_backend.cu:155-188); the
 * solve and one-shot forms extend Backend::Cuda to the solves, which the
 * reference always runs on the CPU (batched.hpp:249, :260). Large batches are
 * streamed through the device in chunks so that the copies overlap the kernels.
 * Memory kept after the call: the first call on a device creates three streams and
 * three device slots sized for its chunk (at most 96 MB of A each, plus B, pivots and
 * info); later calls reuse them and grow them when a chunk needs more. They are kept
 * until the process exits (the uneven-stream host call below keeps its own three
 * slots and pinned record buffers the same way).
 */
int tsdx_cuda_cholesky_batched_host_f32(float* A, int n, int64_t batch, int* info);
int tsdx_cuda_cholesky_batched_host_f64(double* A, int n, int64_t batch, int* info);
int tsdx_cuda_lu_batched_host_f32(float* A, int n, int64_t batch, int* piv, int* info);
int tsdx_cuda_lu_batched_host_f64(double* A, int n, int64_t batch, int* piv, int* info);
int tsdx_cuda_cholesky_solve_batched_host_f32(const float* L, int n, int64_t batch, float* B, int nrhs);
int tsdx_cuda_cholesky_solve_batched_host_f64(const double* L, int n, int64_t batch, double* B, int nrhs);
int tsdx_cuda_lu_solve_batched_host_f32(const float* LU, const int* piv, int n, int64_t batch, float* B, int nrhs);
int tsdx_cuda_lu_solve_batched_host_f64(const double* LU, const int* piv, int n, int64_t batch, double* B, int nrhs);
int tsdx_cuda_posv_batched_host_f32(float* A, int n, int64_t batch, float* B, int nrhs, int* info);
int tsdx_cuda_posv_batched_host_f64(double* A, int n, int64_t batch, double* B, int nrhs, int* info);
int tsdx_cuda_gesv_batched_host_f32(float* A, int n, int64_t batch, float* B, int nrhs, int* piv, int* info);
int tsdx_cuda_gesv_batched_host_f64(double* A, int n, int64_t batch, double* B, int nrhs, int* piv, int* info);

/* One-shot solves that return only (x, info), like the reference's Python-level
 * tsdx.gesv / tsdx.posv (python/tinysolverdx/__init__.py:102-111): A is read and left
 * untouched, B is overwritten by X, no factor or pivots travel back to the host. */
int tsdx_cuda_gesv_solve_host_f32(const float* A, int n, int64_t batch, float* B, int nrhs, int* info);
int tsdx_cuda_gesv_solve_host_f64(const double* A, int n, int64_t batch, double* B, int nrhs, int* info);
int tsdx_cuda_posv_solve_host_f32(const float* A, int n, int64_t batch, float* B, int nrhs, int* info);
int tsdx_cuda_posv_solve_host_f64(const double* A, int n, int64_t batch, double* B, int nrhs, int* info);

/* ---- mixed precision + iterative refinement (no reference counterpart) -------------
 * Solves A x = b (one right-hand side, A (batch, n, n) float64, NOT modified, B (batch, n)
 * float64 overwritten by x) by factoring a power-of-two scaled copy of A in low precision
 * and refining with float64 residuals until the normwise backward error
 * ||b - A x|| / (||A||_F ||x|| + ||b||) (runtime.cpp:230-242) is <= tol or itmax
 * corrections have been applied. Matrices that do not converge are re-solved by the
 * plain float64 kernel in the same call, so every returned x is either refined or fp64.
 *   tier   (batch) int8 per matrix, or NULL to use default_tier for all:
 *          0 fp16 (scaled, tensor cores), 1 bf16 (tensor cores), 2 fp32, 3 fp64 directly
 *   info   (batch) or NULL: fp64 info for fallback matrices, low-precision info otherwise
 *   status (batch) or NULL: refinement steps used (>= 0), or -1 = solved by the fp64 fallback
 *   bwd    (batch) or NULL: the last backward error measured by the refinement
 * gesv_ir pivots (LU); posv_ir assumes A symmetric positive definite (Cholesky).
 */
int tsdx_cuda_gesv_ir_f64(const double* A, int n, int64_t batch, double* B, const signed char* tier,
                          int default_tier, int itmax, double tol, int* info, int* status, double* bwd,
                          void* stream);
int tsdx_cuda_posv_ir_f64(const double* A, int n, int64_t batch, double* B, const signed char* tier,
                          int default_tier, int itmax, double tol, int* info, int* status, double* bwd,
                          void* stream);

/* ---- emulated fp16 / bf16 on the GPU (host pointers, synchronous) -----------------
 * The reference's per-operation-rounding formats (precision.hpp:41-97), which it runs
 * only on the CPU (batched.hpp:130-132), bit-identical to its CPU results. Storage is
 * float64 as in the runtime API (runtime.cpp:95-141); fmt 0 = fp16, 1 = bf16.
 *   factor: lu = 0 Cholesky (A <- L, info), lu = 1 LU (A <- L\U, piv, info)
 *   solve:  lu = 0 B <- (L L^T)^{-1} B, lu = 1 B <- (P L U)^{-1} B */
int tsdx_cuda_emu_factor_host(int fmt, int lu, double* A, int n, int64_t batch, int* piv, int* info);
int tsdx_cuda_emu_solve_host(int fmt, int lu, const double* F, const int* piv, int n, int64_t batch, double* B,
                             int nrhs);

/* ---- error metrics on the GPU ------------------------------------------------------
 * The reference's ground-truth metrics (src/runtime.cpp:194-242, long double on the
 * CPU) computed per matrix in double-double arithmetic on the device; float64
 * inputs, device pointers, out (batch) float64.
 *   solve_backward_error  ||b - A x||_2 / (||A||_F ||x||_2 + ||b||_2)   runtime.cpp:230-242
 *   lu_backward_error     ||P A - L U||_F / ||A||_F  (packed LU, pivots)  runtime.cpp:208-228
 *   chol_backward_error   ||A - L L^T||_F / ||A||_F                      runtime.cpp:194-206 */
int tsdx_cuda_solve_backward_error_f64(const double* A, const double* x, const double* b, int n, int64_t batch,
                                       double* out, void* stream);
int tsdx_cuda_lu_backward_error_f64(const double* A, const double* LU, const int* piv, int n, int64_t batch,
                                    double* out, void* stream);
int tsdx_cuda_chol_backward_error_f64(const double* A, const double* L, int n, int64_t batch, double* out,
                                      void* stream);

/* ---- learned precision-tier selector (no reference counterpart) -------------------
 * A 24 -> 64 -> 64 -> 4 MLP over cheap per-matrix features predicts the cheapest
 * tier (0 fp16, 1 bf16, 2 fp32, 3 fp64) whose refinement converges; the tier array
 * feeds tsdx_cuda_gesv_ir_f64 / tsdx_cuda_posv_ir_f64. All pointers are device
 * pointers, float32 unless stated; the parameter vector (6020 floats) is laid out
 * W1[24][64], b1[64], W2[64][64], b2[64], W3[64][4], b3[4]; norm = mu[24], 1/sd[24].
 *   features: 24 per matrix of the float64 stack A (batch, n, n); kind (batch) int8
 *             0 SPD / 1 general, or NULL to use kind_all for every matrix.
 *   forward:  logits (batch, 4) and/or argmax tier (batch) int8; either may be NULL.
 *   grad:     gradient of sum_s w[y_s] CE_s / batch (class_weight (4) or NULL for 1)
 *             and the loss; scratch >= tsdx_cuda_mlp_scratch_bytes(batch) bytes.
 *   adam:     one Adam step (bias-corrected, step >= 1) on count parameters. */
int tsdx_cuda_selector_features_f64(const double* A, int n, int64_t batch, const signed char* kind, int kind_all,
                                    float* features, void* stream);
int tsdx_cuda_mlp_forward(const float* params, const float* norm, const float* features, int64_t batch,
                          float* logits, signed char* tier, void* stream);
int64_t tsdx_cuda_mlp_scratch_bytes(int64_t batch);
int tsdx_cuda_mlp_grad(const float* params, const float* norm, const float* features, const signed char* label,
                       const float* class_weight, int64_t batch, float* grad, float* loss, void* scratch,
                       int64_t scratch_bytes, void* stream);
int tsdx_cuda_adam_step(float* params, const float* grad, float* m, float* v, int64_t count, float lr,
                        float beta1, float beta2, float eps, int step, void* stream);

/* ---- uneven stream (no reference counterpart) -------------------------------------
 * One call over `count` matrices of mixed order n in [1, 64], Cholesky (kind 0, posv)
 * and LU (kind 1, gesv) mixed, 0..8 right-hand sides each, all in device memory:
 *   A + aoff[i]  n_i x n_i row-major; overwritten by its factor when write_factors != 0
 *   B + boff[i]  n_i x nrhs_i row-major right-hand sides, overwritten by X (B may be NULL)
 *   piv + poff[i] n_i LU pivots (required when write_factors != 0)
 *   info[i]      LAPACK-style info; -1 for an entry outside the supported sizes
 * Factors, pivots, info and X are bit-identical to the dense tsdx_cuda_posv/gesv_*.
 * The matrices are counting-sorted into buckets (kind, padded order, right-hand-side
 * class) and drained by persistent kernels, one per order class of 8 above order 16
 * and one for n <= 16, each through its own atomic queue; the launches are
 * stream-ordered and can be captured in a CUDA graph. sched: bit c (c = 0..3, orders
 * up to 8, 16, 24, 32) runs that class one matrix per warp instead of packing several
 * per warp (8 Cholesky or 4 LU up to order 8, 4 up to 16, 4 (float32) or 2 (float64)
 * up to 24, 2 up to 32); the autotuner of the Python layer chooses it. scratch: device memory of at least
 * tsdx_cuda_stream_scratch_bytes(count) bytes, or NULL to allocate it on the stream. */
int64_t tsdx_cuda_stream_scratch_bytes(int64_t count);
int tsdx_cuda_solve_stream_f32(float* A, const int64_t* aoff, float* B, const int64_t* boff, int* piv,
                               const int64_t* poff, int* info, const int* n, const int* nrhs,
                               const signed char* kind, int64_t count, int write_factors, unsigned sched,
                               void* scratch, int64_t scratch_bytes, void* stream);
int tsdx_cuda_solve_stream_f64(double* A, const int64_t* aoff, double* B, const int64_t* boff, int* piv,
                               const int64_t* poff, int* info, const int* n, const int* nrhs,
                               const signed char* kind, int64_t count, int write_factors, unsigned sched,
                               void* scratch, int64_t scratch_bytes, void* stream);

/* ---- uneven stream from host memory (no reference counterpart) --------------------
 * The same solve with A, B, piv and info in HOST memory, packed back to back in index
 * order: matrix i's A at sum_{j<i} n_j^2 elements, its right-hand sides at
 * sum_{j<i} n_j*nrhs_j, its pivots at sum_{j<i} n_j (the packing of the Python
 * layer's stream.layout). n, nrhs and kind are host arrays too. Synchronous, like the
 * *_batched_host_* calls: the set crosses the device in chunks of about 96 MB (every
 * byte a matrix moves counted), so the device holds three chunks at a time whatever
 * the size of the set, and each chunk's host->device copy overlaps the previous
 * chunk's solve and the device->host copy of the one before. The copies overlap only when the host buffers are pinned
 * (page-locked); pageable buffers work but serialize. Every entry is checked before
 * any copy: n outside [1, 64] -> TSDX_ERR_N, nrhs outside [0, 8] -> TSDX_ERR_NRHS.
 * B may be NULL when every nrhs is 0, piv when write_factors is 0; info may be NULL.
 * The pivot slots of Cholesky matrices come back unchanged.
 * Factors, pivots, info and X are bit-identical to tsdx_cuda_solve_stream_*. */
int tsdx_cuda_solve_stream_host_f32(float* A, float* B, int* piv, int* info, const int* n, const int* nrhs,
                                    const signed char* kind, int64_t count, int write_factors, unsigned sched);
int tsdx_cuda_solve_stream_host_f64(double* A, double* B, int* piv, int* info, const int* n, const int* nrhs,
                                    const signed char* kind, int64_t count, int write_factors, unsigned sched);

/* ---- uneven stream without allocation (no reference counterpart) ------------------
 * tsdx_cuda_solve_stream_f32 with the scratch in a fixed 1 MiB (+520 B) device array
 * of the library instead of caller memory: allocates nothing, for callers that may
 * not allocate device memory at call time (memory owned by another allocator or
 * reserved up front; request paths where cudaMalloc could stall or fail). Every GPU
 * that loads the library keeps the array until exit. At most 262,144
 * matrices per call; a larger count returns TSDX_ERR_TOO_LARGE before any launch.
 * The array's address is looked up once per device on the first call on that device,
 * which must not be made while the stream is being captured, and is kept for the life
 * of the process: it does not survive cudaDeviceReset, so do not call this entry point
 * on a device again after resetting it. The bucket counters
 * that must start at zero are zeroed by every call on its stream. All calls on a
 * device share the array: calls whose executions overlap (other streams or threads)
 * race and corrupt each other's results, so order them (e.g. one stream). */
int tsdx_cuda_solve_stream_noalloc_f32(float* A, const int64_t* aoff, float* B, const int64_t* boff, int* piv,
                                       const int64_t* poff, int* info, const int* n, const int* nrhs,
                                       const signed char* kind, int64_t count, int write_factors,
                                       unsigned sched, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TSDX_CUDA_H */
