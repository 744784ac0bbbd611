// Host-side launchers: map a runtime (n, nrhs) onto a compiled (NP, NRHS) kernel
// and size a persistent grid from the occupancy of that kernel.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "blk.cuh"
#include "solve.cuh"
#include "blk3.cuh"
#include "blk_tc.cuh"

namespace tsdx {
namespace host {

using dev::FastDiv;
using dev::SolveArgs;

// Errors of the CUDA runtime, per calling thread.
void set_cuda_error(cudaError_t e, const char* what);
std::atomic<long long>& launch_counter();

int device_sms(int dev);

// Per-device tables of the library (workspaces, streams, cached addresses) cover
// device ordinals [0, kMaxDevices); a higher ordinal is reported as TSDX_ERR_NODEV.
constexpr int kMaxDevices = 64;

// Compiled padded sizes; a matrix of order n runs in the smallest NP >= n
// (identity padding is exactly transparent to every result, see common.cuh).
inline int np_of(int n) {
  return n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : n <= 24 ? 24 : n <= 32 ? 32 : n <= 40 ? 40 : n <= 48 ? 48 : n <= 56 ? 56 : 64;
}
// Right-hand sides are solved in passes of at most 8 columns.
inline int nrhs_bucket(int r) { return r == 0 ? 0 : r == 1 ? 1 : r <= 4 ? 4 : 8; }
// Widest cp.async chunk that keeps every row start aligned.
template <class T> inline int vec_for(const void* p, int n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const int row = n * int(sizeof(T));
  if (row % 16 == 0 && a % 16 == 0) return 16;
  if (row % 8 == 0 && a % 8 == 0) return 8;
  return 4;
}

template <class Kern>
int grid_for(Kern kern, int smem, long long ctas_needed, int threads = 128) {
  int devi = 0;
  cudaGetDevice(&devi);
  static thread_local int last_dev = -1;
  (void)last_dev;
  int occ = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
  if (e != cudaSuccess || occ < 1) occ = 1;
  const long long cap = (long long)device_sms(devi) * occ;
  return (int)(ctas_needed < cap ? (ctas_needed < 1 ? 1 : ctas_needed) : cap);
}

template <class Kern>
int prepare(Kern kern, int smem) {
  // the attribute is per function and per device; setting it is idempotent
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) { set_cuda_error(e, "cudaFuncSetAttribute"); return -5; }
  }
  return 0;
}

// Blocked LU / Cholesky (blk.cuh): a persistent CTA per SM with as many warps as
// shared memory holds (at most 16).
template <class T, int NP, int NRHS, int GO = 0>
constexpr int blk_wpc() {
  constexpr int FIT = (227 * 1024) / dev::BlkCfg<T, NP, NRHS, GO>::WARPB;
  return FIT < 1 ? 1 : (FIT > 16 ? 16 : FIT);
}

// Lanes per matrix: two matrices share a warp (16 lanes each, two rows per lane)
// where that still leaves 16 warps per SM (orders 17..32 in float32, 17..24 in
// float64) and for float32 LU at order 40. Measured on B200 against one matrix
// per warp at batch 262,144: +12..43 % there, slower wherever it costs warps.
// Orders 9..16 pack four matrices per warp.
template <class T, int NP, int NRHS, bool CHOL>
constexpr int blk_lanes() {
  // order 9..16: four matrices per warp (8 lanes, two rows per lane): +22..50 % over
  // two per warp on B200 at 262,144 matrices (posv fp64 303 -> 405 M solves/s)
  if (NP == 16) return 8;
  // order 5..8 Cholesky: eight per warp (4 lanes): posv 1177 -> 1560 M solves/s (fp64);
  // LU keeps four per warp (the 4-lane LU form is not used)
  if (NP == 8) return CHOL ? 4 : 0;
  // float32 order 17..24: four per warp (8 lanes, three rows per lane): +18 % (posv),
  // +39 % (gesv); float64 keeps two per warp
  if (NP == 24 && sizeof(T) == 4) return 8;
  if (NP <= 16 || NP > 40) return 0;
  if (NP == 40) return (sizeof(T) == 4 && !CHOL) ? 16 : 0;
  return blk_wpc<T, NP, NRHS, 16>() == 16 ? 16 : 0;
}

// Two warps per matrix (blk2.cuh) for float64 LU of padded order 48..56: measured on
// B200 against one warp per matrix at 65,536-131,072 matrices with 4 right-hand
// sides, 1.10x (order 48), 1.22x (56), 1.10x (64); slower at 40 and in float32.
template <class T, int NP, int NRHS>
int launch_blk2(const SolveArgs<T>& a, cudaStream_t st) {
  using C = dev::Blk2Cfg<T, NP, NRHS>;
  constexpr int FIT = (227 * 1024) / C::TEAMB;
  constexpr int TPC = FIT < 1 ? 1 : (FIT > 8 ? 8 : FIT);
  constexpr int SMEM = TPC * C::TEAMB;
  auto kern = dev::blk2_kernel<T, NP, NRHS, TPC>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long ctas = (a.batch + TPC - 1) / TPC;
  const int grid = grid_for(kern, SMEM, ctas, TPC * 64);
  kern<<<grid, TPC * 64, SMEM, st>>>(a);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

// Two warps per matrix with look-ahead (blk3.cuh) for float64 LU of padded order 64:
// 1.10x the two-warp kernel (1.18x at n = 61) on B200, 65,536 matrices, 4 right-hand
// sides; slower than it at orders 40..56.
template <class T, int NP, int NRHS>
int launch_blk3(const SolveArgs<T>& a, cudaStream_t st) {
  using C = dev::Blk3Cfg<T, NP, NRHS>;
  constexpr int FIT = (227 * 1024) / C::TEAMB;
  constexpr int TPC = FIT < 1 ? 1 : (FIT > 8 ? 8 : FIT);
  constexpr int SMEM = TPC * C::TEAMB;
  // the panel warp also takes part of the trailing update (pivot steps counted as 3
  // chunk updates): +3.8 % at n = 64, -1.3 % at n = 61 on B200
  auto kern = dev::blk3_kernel<T, NP, NRHS, TPC, 3>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long ctas = (a.batch + TPC - 1) / TPC;
  const int grid = grid_for(kern, SMEM, ctas, TPC * 64);
  kern<<<grid, TPC * 64, SMEM, st>>>(a);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

// LU kernel family: 0 = by order (the default), 1 = shared-memory blocked kernels
// with CUDA-core updates everywhere (blk.cuh / blk2.cuh / blk3.cuh), 3 = the float64
// tensor-core trailing update (blk_tc.cuh) at every padded order 32..64. Read once
// from TSDX_LU_KERNEL ("smem" or "tc"); all give bit-identical results.
int lu_kernel_family();

// float64 LU with the trailing update on the FP64 tensor cores (blk_tc.cuh): a
// persistent CTA per SM with as many one-matrix warps as shared memory holds.
template <int NP, int NRHS>
int launch_tc(const SolveArgs<double>& a, cudaStream_t st) {
  using C = dev::TcCfg<NP, NRHS>;
  constexpr int FIT = (227 * 1024) / C::WARPB;
  constexpr int WPC = FIT < 1 ? 1 : (FIT > 16 ? 16 : FIT);
  constexpr int SMEM = WPC * C::WARPB;
  auto kern = dev::tc_kernel<NP, NRHS, WPC>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long ctas = (a.batch + WPC - 1) / WPC;
  const int grid = grid_for(kern, SMEM, ctas, WPC * 32);
  kern<<<grid, WPC * 32, SMEM, st>>>(a);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

template <class T, int NP, int NRHS, bool CHOL>
int launch_blk(const SolveArgs<T>& a, cudaStream_t st) {
  // float64 LU from padded order 32 on: the tensor-core trailing update. Measured on
  // B200 against the shared-memory kernels (65,536-262,144 matrices, 4 right-hand
  // sides, M solves/s): n=25 77.1 vs 68.1, n=32 93.0 vs 65.3, n=40 38.0 vs 33.3,
  // n=48 26.8 vs 23.1, n=56 18.2 vs 16.7, n=64 15.3 vs 12.9 (its later changes took
  // n=64 to 16.9: the back substitution, the winner record and U12). Odd orders above 48
  // stay on the shared-memory kernels (n=61 11.6 vs 12.3): their rows are not whole
  // 16-byte units, so the matrix cannot arrive by bulk copies.
  if constexpr (!CHOL && sizeof(T) == 8 && NP >= 32) {
    const int fam = lu_kernel_family();
    if (fam == 3 || (fam == 0 && (NP <= 48 || a.n % 2 == 0)))
      return launch_tc<NP, NRHS>(reinterpret_cast<const SolveArgs<double>&>(a), st);
  }
  if constexpr (!CHOL && sizeof(T) == 8 && NP == 64) return launch_blk3<T, NP, NRHS>(a, st);
  if constexpr (!CHOL && sizeof(T) == 8 && NP >= 48) return launch_blk2<T, NP, NRHS>(a, st);
  constexpr int GO = blk_lanes<T, NP, NRHS, CHOL>();
  using C = dev::BlkCfg<T, NP, NRHS, GO>;
  constexpr int WPC = blk_wpc<T, NP, NRHS, GO>();
  constexpr int SMEM = WPC * C::WARPB;
  auto kern = dev::blk_kernel<T, NP, NRHS, WPC, CHOL, GO>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long units = (a.batch + C::S - 1) / C::S;
  const long long ctas = (units + WPC - 1) / WPC;
  const int grid = grid_for(kern, SMEM, ctas, WPC * 32);
  kern<<<grid, WPC * 32, SMEM, st>>>(a);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

template <class T, int NP, int NRHS, bool LU>
int launch_trs(const SolveArgs<T>& a, int vec, cudaStream_t st) {
  constexpr int SMEM = dev::SolveSmem<T, NP>::CTA;
  auto kern = dev::trs_kernel<T, NP, NRHS, LU>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long ctas = (a.batch + 3) / 4;
  const int grid = grid_for(kern, SMEM, ctas);
  kern<<<grid, 128, SMEM, st>>>(a, FastDiv((unsigned)a.n), vec);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

#define TSDX_NP_SWITCH(NPV, BODY)                 \
  switch (NPV) {                                  \
    case 4: { constexpr int NP_ = 4; BODY; }      \
    case 8: { constexpr int NP_ = 8; BODY; }      \
    case 16: { constexpr int NP_ = 16; BODY; }    \
    case 24: { constexpr int NP_ = 24; BODY; }    \
    case 32: { constexpr int NP_ = 32; BODY; }    \
    case 40: { constexpr int NP_ = 40; BODY; }    \
    case 48: { constexpr int NP_ = 48; BODY; }    \
    case 56: { constexpr int NP_ = 56; BODY; }    \
    default: { constexpr int NP_ = 64; BODY; }    \
  }
#define TSDX_RHS_SWITCH(RV, BODY)                 \
  switch (RV) {                                   \
    case 0: { constexpr int R_ = 0; BODY; }       \
    case 1: { constexpr int R_ = 1; BODY; }       \
    case 4: { constexpr int R_ = 4; BODY; }       \
    default: { constexpr int R_ = 8; BODY; }      \
  }

// One fused pass: factor A (and solve B columns [b0, b0 + nrhs), nrhs <= 8).
template <class T, bool CHOL>
int run_blk(const SolveArgs<T>& a, cudaStream_t st) {
  const int np = np_of(a.n), rb = nrhs_bucket(a.nrhs);
  TSDX_NP_SWITCH(np, TSDX_RHS_SWITCH(rb, return (launch_blk<T, NP_, R_, CHOL>(a, st))));
  return 0;
}

// One solve pass from a factor (nrhs <= 8).
template <class T, bool LU>
int run_trs(const SolveArgs<T>& a, cudaStream_t st) {
  const int vec = vec_for<T>(a.A, a.n);
  SolveArgs<T> b = a;
  b.rowdiv = FastDiv((unsigned)(a.n * int(sizeof(T)) / vec));
  const int np = np_of(a.n) <= 32 ? 32 : 64, rb = nrhs_bucket(a.nrhs);
  if (np == 32) {
    TSDX_RHS_SWITCH(rb == 0 ? 1 : rb, return (launch_trs<T, 32, (R_ > 0 ? R_ : 1), LU>(b, vec, st)));
  }
  TSDX_RHS_SWITCH(rb == 0 ? 1 : rb, return (launch_trs<T, 64, (R_ > 0 ? R_ : 1), LU>(b, vec, st)));
  return 0;
}

// Explicitly instantiated in the per-type translation units.
template <class T> int run_lu(const SolveArgs<T>& a, cudaStream_t st);
template <class T> int run_chol(const SolveArgs<T>& a, cudaStream_t st);
template <class T> int run_getrs(const SolveArgs<T>& a, cudaStream_t st);
template <class T> int run_potrs(const SolveArgs<T>& a, cudaStream_t st);

}  // namespace host
}  // namespace tsdx
