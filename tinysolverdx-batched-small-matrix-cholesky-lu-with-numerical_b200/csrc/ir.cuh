// Mixed-precision factorization + fp64 iterative refinement (gesv_ir / posv_ir).
//
// No reference counterpart: TinySolverDx only emulates fp16/bf16 on the CPU
// (precision.hpp:71-97). Per matrix (one warp, persistent CTA rounds):
//   1. A (fp64, global) is read once, coalesced, and written to shared memory as
//      an fp32 working matrix, scaled by powers of two (rows then columns, max
//      |a| -> 1, exact) so fp16 tensor-core operands stay in range.
//   2. The scaled matrix is factored in fp32 with partial pivoting (LU) or, for
//      symmetric positive definite input, without pivoting (A = L U with U = D L^T,
//      the Cholesky factor up to a diagonal: SPD matrices need no pivoting, and the
//      shared code keeps one fast path): 16-column panels in registers, the trailing update
//      A22 -= L21 U12 either on the tensor cores (mma.sync m16n8k16, fp16 or bf16
//      operands, fp32 accumulation) or on the fp32 CUDA cores, by tier.
//   3. x0 = A^{-1} b with the low-precision factors (fp32 triangular solves,
//      reciprocal pivots computed once after the factorization).
//   4. Refinement: r = b - A x in fp64 straight from A in global memory (rows
//      read coalesced, 32 row sums per lane folded by a transposing butterfly),
//      normwise backward error ||r|| / (||A||_F ||x|| + ||b||)
//      (runtime.cpp:230-242); stop when it is <= tol, else x += A^{-1} r with the
//      same factors.
// A matrix that does not converge within itmax steps (or meets a zero / non-
// positive pivot in low precision) is reported with status -1; the host then
// solves it with the plain fp64 kernel (the fallback is never silent).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace tsdx {
namespace dev {

struct IrArgs {
  const double* A;            // (batch, n, n), not modified
  double* B;                  // (batch, n): right-hand side in, solution out
  int* info;                  // (batch) low-precision factorization info, or nullptr
  const signed char* tier;    // (batch) per-matrix tier, or nullptr -> default_tier
  int* status;                // (batch) refinement steps used, -1 = not converged
  double* bwd;                // (batch) final normwise backward error, or nullptr
  const int* idx;             // optional (batch) list of matrix indices to solve
  long long batch;
  int n, default_tier, itmax;
  double tol;
};

enum Tier { kTierF16 = 0, kTierBF16 = 1, kTierF32 = 2, kTierF64 = 3 };

__device__ __forceinline__ unsigned pack2(float lo, float hi, bool f16) {
  if (f16) {
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&h);
  }
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&h);
}

// D = A(16x16) * B(16x8) + C, fp32 accumulation; A row-major, B column-major fragments.
__device__ __forceinline__ void mma16816(float* d, const unsigned* a, const unsigned* b, bool f16) {
  if (f16)
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
  else
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int NP>
struct IrCfg {
  static constexpr int MR = (NP + 31) / 32;
  static constexpr int PB = 16;
  static constexpr int RSF = NP * 4 + 16;  // fp32 row: an odd number of 16-byte units
  static constexpr int F = NP * RSF;
  // ord (int), x (double), column scales, row scales, reciprocal pivots (float)
  static constexpr int AUX = NP * 4 + NP * 8 + NP * 4 * 3 + 32;
  static constexpr int WARPB = (F + AUX + 127) / 128 * 128;
  // cooperative float4 passes: CG groups of 4 columns, RPI rows per pass
  static constexpr int CG = NP / 4;
  static constexpr int CGP = CG <= 4 ? 4 : CG <= 8 ? 8 : 16;
  static constexpr int RPI = 32 / CGP;
  static_assert(NP % 16 == 0, "tensor-core tiles need NP % 16 == 0");
};

template <int NP, bool SPD, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) ir_kernel(IrArgs p) {
  using C = IrCfg<NP>;
  constexpr int MR = C::MR, PB = C::PB, RSF = C::RSF, CG = C::CG, CGP = C::CGP, RPI = C::RPI;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* Fb = smem + warp * C::WARPB;
  int* ord = reinterpret_cast<int*>(Fb + C::F);
  double* xs = reinterpret_cast<double*>(Fb + C::F + NP * 4);
  float* csc = reinterpret_cast<float*>(Fb + C::F + NP * 12);
  float* rsd = csc + NP;
  float* rinv = rsd + NP;
  auto F = [&](int r, int c) -> float& { return *reinterpret_cast<float*>(Fb + r * RSF + c * 4); };
  auto F4 = [&](int r, int c) -> float4& { return *reinterpret_cast<float4*>(Fb + r * RSF + c * 4); };
  const int n = p.n;
  const long long per_round = (long long)gridDim.x * WPC;
  const int q4 = lane % CGP, rho = lane / CGP;  // cooperative pass coordinates

  for (long long base = (long long)blockIdx.x * WPC; base < p.batch; base += per_round) {
    __syncthreads();
    const long long t = base + warp;
    if (t >= p.batch) continue;
    const long long m = p.idx ? (long long)p.idx[t] : t;
    const int tier = p.tier ? (int)p.tier[m] : p.default_tier;
    if (tier >= kTierF64) {  // solved directly by the fp64 pass
      if (lane == 0 && p.status) p.status[m] = -1;
      continue;
    }
    const bool tc = tier == kTierF16 || tier == kTierBF16;
    const bool f16 = tier == kTierF16;
    const double* Ag = p.A + m * (long long)n * n;
    double* Bg = p.B + m * (long long)n;

    // ------------------------------------------ 1. load, scale, ||A||_F, b
    double afro = 0.0;
    float rsc[MR];
    {
      // coalesced row reads (lane c holds columns c, c + 32), unscaled fp32 copy
#pragma unroll 4
      for (int r = 0; r < n; ++r) {
        const double* row = Ag + (long long)r * n;
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int c = lane + 32 * s;
          if (c < n) {
            const double v = __ldg(row + c);
            afro = fma(v, v, afro);
            F(r, c) = (float)v;
          }
        }
      }
      if (n < NP) {  // identity padding
        for (int r = 0; r < NP; ++r)
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int c = lane + 32 * s;
            if (c < NP && (r >= n || c >= n)) F(r, c) = (r == c) ? 1.f : 0.f;
          }
      }
      for (int o = 16; o > 0; o >>= 1) afro += __shfl_xor_sync(kFull, afro, o);
      __syncwarp();
      // row scales: each lane scans its own rows with 16-byte reads
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        float mx = 0.f;
        if (r < n) {
#pragma unroll
          for (int c = 0; c < NP; c += 4) {
            const float4 v = F4(r, c);
            mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
          }
        }
        int e = 0;
        frexpf(mx, &e);
        rsc[s] = (r < n && mx > 0.f && isfinite(mx)) ? ldexpf(1.f, -e) : 1.f;
        if (r < NP) rsd[r] = rsc[s];
      }
      __syncwarp();
      // apply the row scales and take column maxima (lanes: 4 columns x RPI rows)
      float cm[4] = {0.f, 0.f, 0.f, 0.f};
      if (q4 < CG) {
        for (int r = rho; r < NP; r += RPI) {
          float4 v = F4(r, 4 * q4);
          const float sc = rsd[r];
          v.x *= sc; v.y *= sc; v.z *= sc; v.w *= sc;
          F4(r, 4 * q4) = v;
          cm[0] = fmaxf(cm[0], fabsf(v.x));
          cm[1] = fmaxf(cm[1], fabsf(v.y));
          cm[2] = fmaxf(cm[2], fabsf(v.z));
          cm[3] = fmaxf(cm[3], fabsf(v.w));
        }
      }
#pragma unroll
      for (int o = CGP; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < 4; ++i) cm[i] = fmaxf(cm[i], __shfl_xor_sync(kFull, cm[i], o));
      if (rho == 0 && q4 < CG) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int c = 4 * q4 + i;
          int e = 0;
          frexpf(cm[i], &e);
          // SPD keeps symmetry: D A D with D the row scales
          const float cs = SPD ? rsd[c] : ((c < n && cm[i] > 0.f && isfinite(cm[i])) ? ldexpf(1.f, -e) : 1.f);
          csc[c] = cs;
        }
      }
      __syncwarp();
      if (q4 < CG) {
        const float4 cs = *reinterpret_cast<const float4*>(csc + 4 * q4);
        for (int r = rho; r < NP; r += RPI) {
          float4 v = F4(r, 4 * q4);
          v.x *= cs.x; v.y *= cs.y; v.z *= cs.z; v.w *= cs.w;
          F4(r, 4 * q4) = v;
        }
      }
      __syncwarp();
    }
    double bv[MR];
    double bnrm = 0.0;
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      bv[s] = (r < n) ? Bg[r] : 0.0;
      bnrm = fma(bv[s], bv[s], bnrm);
    }
    for (int o = 16; o > 0; o >>= 1) bnrm += __shfl_xor_sync(kFull, bnrm, o);
    afro = sqrt(afro);
    bnrm = sqrt(bnrm);

    // ------------------------------------------------ 2. low-precision factor
    int pos[MR];
    bool act[MR];
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      act[s] = r < NP;
      pos[s] = r < NP ? r : 0x3fffffff;
    }
    int info = 0;
    for (int k0 = 0; k0 < NP; k0 += PB) {
      float pan[MR][PB];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int rr = (lane + 32 * s < NP) ? lane + 32 * s : 0;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += 4) {
          const float4 v = F4(rr, k0 + i0);
          pan[s][i0] = v.x; pan[s][i0 + 1] = v.y; pan[s][i0 + 2] = v.z; pan[s][i0 + 3] = v.w;
        }
      }
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int k = k0 + i;
        {
          int bpos = k;  // SPD: no pivoting (A = L U with U = D L^T)
          if (!SPD) {
          unsigned bk = 0;
          int bp = 0x7fffffff;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const unsigned key = act[s] ? __float_as_uint(fabsf(pan[s][i])) + 1u : 0u;
            const bool better = key > bk || (key == bk && pos[s] < bp);
            bk = (act[s] && better) ? key : bk;
            bp = (act[s] && better) ? pos[s] : bp;
          }
          const unsigned mk = __reduce_max_sync(kFull, bk);
          bpos = __reduce_min_sync(kFull, bk == mk ? bp : 0x7fffffff);
          }
          int myslot = -1;
#pragma unroll
          for (int s = 0; s < MR; ++s) myslot = (act[s] && pos[s] == bpos) ? s : myslot;
          const int wl = __ffs(__ballot_sync(kFull, myslot >= 0)) - 1;
          const int wslot = MR > 1 ? __shfl_sync(kFull, myslot, wl) : 0;
          float uw[PB];
#pragma unroll
          for (int j = i; j < PB; ++j) {
            float v = pan[0][j];
#pragma unroll
            for (int t2 = 1; t2 < MR; ++t2) v = (wslot == t2) ? pan[t2][j] : v;
            uw[j] = __shfl_sync(kFull, v, wl);
          }
          if (lane == wl) ord[k] = lane + 32 * wslot;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const bool win = act[s] && pos[s] == bpos;
            const bool atk = act[s] && !win && pos[s] == k;
            pos[s] = win ? k : (atk ? bpos : pos[s]);
            act[s] = act[s] && !win;
          }
          const bool zero = SPD ? (!(uw[i] > 0.f) || !isfinite(uw[i])) : (!(uw[i] != 0.f) || !isfinite(uw[i]));
          if (zero && info == 0) info = k + 1;
          const float ry = zero ? 0.f : 1.f / uw[i];
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            if (!act[s]) continue;
            const float l = pan[s][i] * ry;
            pan[s][i] = l;
#pragma unroll
            for (int j = i + 1; j < PB; ++j) pan[s][j] = fmaf(-l, uw[j], pan[s][j]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        if (r >= NP) continue;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += 4)
          F4(r, k0 + i0) = make_float4(pan[s][i0], pan[s][i0 + 1], pan[s][i0 + 2], pan[s][i0 + 3]);
      }
      __syncwarp();
      const int j1 = k0 + PB;
      if (j1 >= NP) continue;
      int ordp[PB];  // physical rows of the panel's pivots
#pragma unroll
      for (int i = 0; i < PB; ++i) ordp[i] = ord[k0 + i];
      {
        // U12: the panel's pivot rows on the trailing columns (unit-lower solve)
        for (int j = j1 + lane; j < NP; j += 32) {
          float u[PB];
#pragma unroll
          for (int i = 0; i < PB; ++i) {
            float acc = F(ordp[i], j);
#pragma unroll
            for (int i2 = 0; i2 < i; ++i2) acc = fmaf(-F(ordp[i], k0 + i2), u[i2], acc);
            u[i] = acc;
            if (i > 0) F(ordp[i], j) = acc;
          }
        }
        __syncwarp();
      }
      // trailing update of the rows still active
      if (tc) {
        const int g = lane >> 2, tq = lane & 3;
#pragma unroll
        for (int rt = 0; rt < NP / 16; ++rt) {
          const int ra = rt * 16 + g, rb = ra + 8;
          // rows still being updated: those not yet retired
          bool sa, sb;
          {
            int va = act[0], vb = act[0];
#pragma unroll
            for (int t2 = 1; t2 < MR; ++t2) {
              va = ((ra >> 5) == t2) ? (int)act[t2] : va;
              vb = ((rb >> 5) == t2) ? (int)act[t2] : vb;
            }
            sa = __shfl_sync(kFull, va, ra & 31) != 0;
            sb = __shfl_sync(kFull, vb, rb & 31) != 0;
          }
          // L21 fragment (negated): rows ra/rb, panel columns k0 + [2tq, 2tq+1, 2tq+8, 2tq+9]
          unsigned af[4];
          af[0] = pack2(-F(ra, k0 + 2 * tq), -F(ra, k0 + 2 * tq + 1), f16);
          af[1] = pack2(-F(rb, k0 + 2 * tq), -F(rb, k0 + 2 * tq + 1), f16);
          af[2] = pack2(-F(ra, k0 + 2 * tq + 8), -F(ra, k0 + 2 * tq + 9), f16);
          af[3] = pack2(-F(rb, k0 + 2 * tq + 8), -F(rb, k0 + 2 * tq + 9), f16);
          for (int ct = j1 / 8; ct < NP / 8; ++ct) {
            const int c0 = ct * 8 + 2 * tq;
            // U12 fragment: B[k][n] = U(k0+k, col ct*8+g)
            unsigned bf[2];
            const int cg = ct * 8 + g;
            bf[0] = pack2(F(ord[k0 + 2 * tq], cg), F(ord[k0 + 2 * tq + 1], cg), f16);
            bf[1] = pack2(F(ord[k0 + 2 * tq + 8], cg), F(ord[k0 + 2 * tq + 9], cg), f16);
            float d[4] = {F(ra, c0), F(ra, c0 + 1), F(rb, c0), F(rb, c0 + 1)};
            mma16816(d, af, bf, f16);
            if (sa) { F(ra, c0) = d[0]; F(ra, c0 + 1) = d[1]; }
            if (sb) { F(rb, c0) = d[2]; F(rb, c0 + 1) = d[3]; }
          }
        }
      } else {
        // fp32 CUDA-core update, 8 columns at a time; each pivot-row segment is read
        // once for all of a lane's rows
        for (int jc = j1; jc < NP; jc += 8) {
          float acc[MR][8];
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = (lane + 32 * s < NP) ? lane + 32 * s : 0;
            const float4 a0 = F4(r, jc), a1 = F4(r, jc + 4);
            acc[s][0] = a0.x; acc[s][1] = a0.y; acc[s][2] = a0.z; acc[s][3] = a0.w;
            acc[s][4] = a1.x; acc[s][5] = a1.y; acc[s][6] = a1.z; acc[s][7] = a1.w;
          }
#pragma unroll
          for (int i = 0; i < PB; ++i) {
            float u[8];
            const float4 v0 = F4(ordp[i], jc), v1 = F4(ordp[i], jc + 4);
            u[0] = v0.x; u[1] = v0.y; u[2] = v0.z; u[3] = v0.w;
            u[4] = v1.x; u[5] = v1.y; u[6] = v1.z; u[7] = v1.w;
#pragma unroll
            for (int s = 0; s < MR; ++s)
#pragma unroll
              for (int q = 0; q < 8; ++q) acc[s][q] = fmaf(-pan[s][i], u[q], acc[s][q]);
          }
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lane + 32 * s;
            const bool on = act[s] && r < NP;
            if (!on) continue;
            F4(r, jc) = make_float4(acc[s][0], acc[s][1], acc[s][2], acc[s][3]);
            F4(r, jc + 4) = make_float4(acc[s][4], acc[s][5], acc[s][6], acc[s][7]);
          }
        }
      }
      __syncwarp();
    }
    if (p.info && lane == 0) p.info[m] = info;
    // reciprocal pivots U(ord[k], k)
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int k = lane + 32 * s;
      if (k < NP) rinv[k] = 1.f / F(ord[k], k);
    }
    __syncwarp();

    // ---------------------------------------- 3./4. solve and refine in fp64
    // lowsolve(v): v = D_r * rhs by physical row in; the scaled solution by physical row out
    auto lowsolve = [&](float* v) {
      // forward: y_k at physical row ord[k]; rows retired after k take -L(row,k) y_k
      for (int k = 0; k < NP; ++k) {
        const int pk = ord[k];
        float vk = v[0];
#pragma unroll
        for (int t2 = 1; t2 < MR; ++t2) vk = ((pk >> 5) == t2) ? v[t2] : vk;
        const float y = __shfl_sync(kFull, vk, pk & 31);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          if (pos[s] > k && r < NP) v[s] = fmaf(-F(r, k), y, v[s]);
        }
      }
      // backward: x_k = y_k / U(ord[k],k); rows retired before k take -U(row,k) x_k
      for (int k = NP - 1; k >= 0; --k) {
        const int pk = ord[k];
        float vk = v[0];
#pragma unroll
        for (int t2 = 1; t2 < MR; ++t2) vk = ((pk >> 5) == t2) ? v[t2] : vk;
        const float x = __shfl_sync(kFull, vk, pk & 31) * rinv[k];
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          if (r == pk) v[s] = x;
          else if (pos[s] < k && r < NP) v[s] = fmaf(-F(r, k), x, v[s]);
        }
      }
      __syncwarp();
    };
    // the solution component of unknown pos[s] sits at physical row r; unscale into xs
    auto gather = [&](const float* v, bool add) {
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        if (r >= NP) continue;
        const int kk = pos[s];
        const double xk = (double)v[s] * (double)csc[kk];
        if (kk < n) xs[kk] = add ? xs[kk] + xk : xk;
      }
      __syncwarp();
    };
    // r = b - A x for the lane's rows lane + 32 s. Rows are read coalesced (lane c
    // multiplies columns c, c + 32) in chunks of 16; a transposing butterfly folds the
    // 16 partial sums of each lane so that lanes 2i and 2i + 1 both end with row
    // 16 ch + i, and one shuffle per chunk hands each row to its owning lane.
    auto residual = [&](double* rr) {
      constexpr int NCH = NP / 16;
      double xl[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int c = lane + 32 * s;
        xl[s] = (c < n) ? xs[c] : 0.0;
      }
      double cv[NCH];
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        double pp[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int r = 16 * ch + j;
          double acc = 0.0;
          if (r < n) {
            const double* row = Ag + (long long)r * n;
#pragma unroll
            for (int s = 0; s < MR; ++s) {
              const int c = lane + 32 * s;
              if (c < n) acc = fma(__ldg(row + c), xl[s], acc);
            }
          }
          pp[j] = acc;
        }
#pragma unroll
        for (int o = 16, w = 8; w >= 1; o >>= 1, w >>= 1) {
          const bool up = (lane & o) != 0;
#pragma unroll
          for (int j = 0; j < w; ++j) {
            const double send = up ? pp[j] : pp[j + w];
            const double keep = up ? pp[j + w] : pp[j];
            pp[j] = keep + __shfl_xor_sync(kFull, send, o);
          }
        }
        cv[ch] = pp[0] + __shfl_xor_sync(kFull, pp[0], 1);
      }
      // row lane + 32 s is row (lane & 15) of chunk 2 s + (lane >> 4) (chunk 0 only for NP = 16)
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        const double a = __shfl_sync(kFull, cv[(2 * s) < NCH ? 2 * s : NCH - 1], 2 * (lane & 15));
        const double b = __shfl_sync(kFull, cv[(2 * s + 1) < NCH ? 2 * s + 1 : NCH - 1], 2 * (lane & 15));
        const double sum = (lane >> 4) ? b : a;
        rr[s] = (r < n) ? bv[s] - sum : 0.0;
      }
    };
    float v[MR];
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      v[s] = (r < n) ? (float)(bv[s] * (double)rsc[s]) : 0.f;
    }
    lowsolve(v);
    gather(v, false);
    int steps = 0;
    double be = 1.0, be_prev = 1e300;
    bool conv = false;
    for (int it = 0; it <= p.itmax + 1; ++it) {
      double rr[MR];
      residual(rr);
      double rn = 0.0, xn = 0.0;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        rn = fma(rr[s], rr[s], rn);
        const int c = lane + 32 * s;
        if (c < n) xn = fma(xs[c], xs[c], xn);
      }
      for (int o = 16; o > 0; o >>= 1) {
        rn += __shfl_xor_sync(kFull, rn, o);
        xn += __shfl_xor_sync(kFull, xn, o);
      }
      be = sqrt(rn) / (afro * sqrt(xn) + bnrm);
      // converged once below tol AND at the fp64 floor: the last correction no longer
      // halved the backward error (or it is already below a quarter unit roundoff)
      if (be <= p.tol && (be > 0.5 * be_prev || be <= 0x1p-55)) { conv = true; break; }
      if (info != 0 || !(be < be_prev)) { conv = be <= p.tol; break; }
      if (steps == p.itmax + (be <= p.tol ? 1 : 0)) { conv = be <= p.tol; break; }
      be_prev = be;
      ++steps;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        v[s] = (r < n) ? (float)(rr[s] * (double)rsc[s]) : 0.f;
      }
      lowsolve(v);
      gather(v, true);
    }
    if (lane == 0) {
      if (p.status) p.status[m] = (conv && info == 0) ? steps : -1;
      if (p.bwd) p.bwd[m] = be;
    }
    if (conv && info == 0)
      for (int c = lane; c < n; c += 32) Bg[c] = xs[c];
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace tsdx
