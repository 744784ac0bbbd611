// Mixed-precision + iterative-refinement solves (ir.cuh) and their fp64 fallback.
#include <cuda_runtime.h>

#include <algorithm>

#include "ir.cuh"
#include "launch.cuh"

namespace tsdx {
namespace host {

template <int NP, bool SPD>
int launch_ir(const dev::IrArgs& a, cudaStream_t st) {
  using C = dev::IrCfg<NP>;
  // at most 12 warps from order 32 up: 170 registers per thread keep the panel,
  // the trailing-update accumulators and the residual butterfly out of local memory
  constexpr int FIT = (227 * 1024) / C::WARPB;
  constexpr int CAP = NP >= 32 ? 12 : 16;
  constexpr int WPC = FIT < 1 ? 1 : (FIT > CAP ? CAP : FIT);
  constexpr int SMEM = WPC * C::WARPB;
  auto kern = dev::ir_kernel<NP, SPD, WPC>;
  if (int rc = prepare(kern, SMEM)) return rc;
  const long long ctas = (a.batch + WPC - 1) / WPC;
  const int grid = grid_for(kern, SMEM, ctas, WPC * 32);
  kern<<<grid, WPC * 32, SMEM, st>>>(a);
  launch_counter().fetch_add(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(e, "kernel launch"); return -5; }
  return 0;
}

// Low-precision factor + refinement over the whole batch, then the plain fp64
// kernel on exactly the matrices whose refinement did not converge (status < 0).
int run_ir(bool spd, const double* A, int n, long long batch, double* B, const signed char* tier, int default_tier,
           int itmax, double tol, int* info, int* status, double* bwd, cudaStream_t st) {
  dev::IrArgs a{};
  a.A = A;
  a.B = B;
  a.info = info;
  a.tier = tier;
  a.status = status;
  a.bwd = bwd;
  a.idx = nullptr;
  a.batch = batch;
  a.n = n;
  a.default_tier = default_tier;
  a.itmax = itmax;
  a.tol = tol;
  const int np = n <= 16 ? 16 : n <= 32 ? 32 : n <= 48 ? 48 : 64;
  int rc = 0;
  switch (np) {
    case 16: rc = spd ? launch_ir<16, true>(a, st) : launch_ir<16, false>(a, st); break;
    case 32: rc = spd ? launch_ir<32, true>(a, st) : launch_ir<32, false>(a, st); break;
    case 48: rc = spd ? launch_ir<48, true>(a, st) : launch_ir<48, false>(a, st); break;
    default: rc = spd ? launch_ir<64, true>(a, st) : launch_ir<64, false>(a, st); break;
  }
  if (rc) return rc;
  dev::SolveArgs<double> f{};
  f.A = const_cast<double*>(A);
  f.B = B;
  f.piv = nullptr;
  f.info = info;
  f.batch = batch;
  f.n = n;
  f.ldb = 1;
  f.b0 = 0;
  f.nrhs = 1;
  f.status = status;
  f.wf = 0;
  return spd ? run_chol<double>(f, st) : run_lu<double>(f, st);
}

}  // namespace host
}  // namespace tsdx
