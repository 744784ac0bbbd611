// Host-pointer C-ABI of the emulated fp16 / bf16 path (emu.cuh): copy in, one
// thread per matrix, copy out, synchronous, like the *_batched_host_* family.
#include <cuda_runtime.h>

#include "../../include/tsdx_cuda.h"
#include "emu.cuh"
#include "launch.cuh"

#define API extern "C" __attribute__((visibility("default")))

namespace {
using namespace tsdx;

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

int fail(cudaError_t e, const char* what) {
  host::set_cuda_error(e, what);
  return TSDX_ERR_CUDA;
}

#define EMU_TRY(call, what)                  \
  do {                                       \
    const cudaError_t e_ = (call);           \
    if (e_ != cudaSuccess) return fail(e_, what); \
  } while (0)

int check(int fmt, int n, int64_t batch) {
  if (fmt != 0 && fmt != 1) return TSDX_ERR_NULL;
  if (n < 1 || n > 64) return TSDX_ERR_N;
  if (batch < 0) return TSDX_ERR_BATCH;
  int dev = 0;
  if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) {
    cudaGetLastError();
    return TSDX_ERR_NODEV;
  }
  return TSDX_OK;
}

unsigned blocks(int64_t batch) { return (unsigned)((batch + 127) / 128); }

int done(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e, what);
  host::launch_counter().fetch_add(1);
  return TSDX_OK;
}
}  // namespace

API int tsdx_cuda_emu_factor_host(int fmt, int lu, double* A, int n, int64_t batch, int* piv, int* info) {
  if (int rc = check(fmt, n, batch)) return rc;
  if (batch == 0) return TSDX_OK;
  if (!A || (lu && !piv)) return TSDX_ERR_NULL;
  const size_t na = (size_t)batch * n * n * sizeof(double), np = (size_t)batch * n * sizeof(int),
               ni = (size_t)batch * sizeof(int);
  DevBuf dA, dP, dI;
  EMU_TRY(cudaMalloc(&dA.p, na), "cudaMalloc");
  EMU_TRY(cudaMalloc(&dI.p, ni), "cudaMalloc");
  if (lu) EMU_TRY(cudaMalloc(&dP.p, np), "cudaMalloc");
  EMU_TRY(cudaMemcpy(dA.p, A, na, cudaMemcpyHostToDevice), "cudaMemcpy");
  double* a = static_cast<double*>(dA.p);
  int* p = static_cast<int*>(dP.p);
  int* in = static_cast<int*>(dI.p);
  if (lu) {
    if (fmt == 0) dev::emu_lu_kernel<0><<<blocks(batch), 128>>>(a, n, batch, p, in);
    else dev::emu_lu_kernel<1><<<blocks(batch), 128>>>(a, n, batch, p, in);
  } else {
    if (fmt == 0) dev::emu_cholesky_kernel<0><<<blocks(batch), 128>>>(a, n, batch, in);
    else dev::emu_cholesky_kernel<1><<<blocks(batch), 128>>>(a, n, batch, in);
  }
  if (int rc = done("emulated factor kernel")) return rc;
  EMU_TRY(cudaMemcpy(A, a, na, cudaMemcpyDeviceToHost), "cudaMemcpy");
  if (lu) EMU_TRY(cudaMemcpy(piv, p, np, cudaMemcpyDeviceToHost), "cudaMemcpy");
  if (info) EMU_TRY(cudaMemcpy(info, in, ni, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return TSDX_OK;
}

API int tsdx_cuda_emu_solve_host(int fmt, int lu, const double* F, const int* piv, int n, int64_t batch, double* B,
                                 int nrhs) {
  if (int rc = check(fmt, n, batch)) return rc;
  if (nrhs < 0) return TSDX_ERR_NRHS;
  if (batch == 0 || nrhs == 0) return TSDX_OK;
  if (!F || !B || (lu && !piv)) return TSDX_ERR_NULL;
  const size_t nf = (size_t)batch * n * n * sizeof(double), nb = (size_t)batch * n * nrhs * sizeof(double),
               np = (size_t)batch * n * sizeof(int);
  DevBuf dF, dB, dP;
  EMU_TRY(cudaMalloc(&dF.p, nf), "cudaMalloc");
  EMU_TRY(cudaMalloc(&dB.p, nb), "cudaMalloc");
  if (lu) EMU_TRY(cudaMalloc(&dP.p, np), "cudaMalloc");
  EMU_TRY(cudaMemcpy(dF.p, F, nf, cudaMemcpyHostToDevice), "cudaMemcpy");
  EMU_TRY(cudaMemcpy(dB.p, B, nb, cudaMemcpyHostToDevice), "cudaMemcpy");
  if (lu) EMU_TRY(cudaMemcpy(dP.p, piv, np, cudaMemcpyHostToDevice), "cudaMemcpy");
  const double* f = static_cast<const double*>(dF.p);
  const int* p = static_cast<const int*>(dP.p);
  double* b = static_cast<double*>(dB.p);
  if (lu) {
    if (fmt == 0) dev::emu_solve_kernel<0, true><<<blocks(batch), 128>>>(f, p, n, batch, b, nrhs);
    else dev::emu_solve_kernel<1, true><<<blocks(batch), 128>>>(f, p, n, batch, b, nrhs);
  } else {
    if (fmt == 0) dev::emu_solve_kernel<0, false><<<blocks(batch), 128>>>(f, nullptr, n, batch, b, nrhs);
    else dev::emu_solve_kernel<1, false><<<blocks(batch), 128>>>(f, nullptr, n, batch, b, nrhs);
  }
  if (int rc = done("emulated solve kernel")) return rc;
  EMU_TRY(cudaMemcpy(B, b, nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return TSDX_OK;
}
