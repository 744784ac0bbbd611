// Mixed-precision factorization + fp64 iterative refinement (gesv_ir / posv_ir).
//
// No reference counterpart: TinySolverDx only emulates fp16/bf16 on the CPU
// (precision.hpp:71-97). Per matrix (one warp, persistent CTA rounds):
//   1. A (fp64, global) is read once, coalesced, and written to shared memory as
//      an fp32 working matrix, scaled by powers of two (rows then columns, max
//      |a| -> 1, exact) so fp16 tensor-core operands stay in range.
//   2. The scaled matrix is factored in fp32 with partial pivoting (LU) or
//      without (Cholesky): 16-column panels in registers, the trailing update
//      A22 -= L21 U12 either on the tensor cores (mma.sync m16n8k16, fp16 or bf16
//      operands, fp32 accumulation) or on the fp32 CUDA cores, by tier.
//   3. x0 = A^{-1} b with the low-precision factors (fp32 triangular solves).
//   4. Refinement: r = b - A x in fp64 straight from A in global memory, normwise
//      backward error ||r|| / (||A||_F ||x|| + ||b||) (runtime.cpp:230-242); stop
//      when it is <= tol, else x += A^{-1} r with the same factors.
// A matrix that does not converge within itmax steps (or meets a zero / non-
// positive pivot in low precision) is reported with status -1; the host then
// solves it with the plain fp64 kernel (the fallback is never silent).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "team.cuh"

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
  static constexpr int AUX = NP * 4 /*ord*/ + NP * 8 /*x*/ + NP * 4 /*col scale*/ + 32;
  static constexpr int WARPB = (F + AUX + 127) / 128 * 128;
  static_assert(NP % 16 == 0, "tensor-core tiles need NP % 16 == 0");
};

template <int NP, bool SPD, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) ir_kernel(IrArgs p) {
  using C = IrCfg<NP>;
  constexpr int MR = C::MR, PB = C::PB, RSF = C::RSF;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* Fb = smem + warp * C::WARPB;
  int* ord = reinterpret_cast<int*>(Fb + C::F);
  double* xs = reinterpret_cast<double*>(Fb + C::F + NP * 4);
  float* csc = reinterpret_cast<float*>(Fb + C::F + NP * 12);
  auto F = [&](int r, int c) -> float& { return *reinterpret_cast<float*>(Fb + r * RSF + c * 4); };
  auto F4 = [&](int r, int c) -> float4& { return *reinterpret_cast<float4*>(Fb + r * RSF + c * 4); };
  const int n = p.n;
  const long long per_round = (long long)gridDim.x * WPC;

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
      // row scales: lane r holds rows r, r+32; one coalesced row read per step
      float rmax[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) rmax[s] = 0.f;
      for (int r = 0; r < n; ++r) {
        const double* row = Ag + (long long)r * n;
        float mx = 0.f;
        for (int c = lane; c < n; c += 32) {
          const double v = row[c];
          afro = fma(v, v, afro);
          mx = fmaxf(mx, (float)fabs(v));
          F(r, c) = (float)v;
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
#pragma unroll
        for (int s = 0; s < MR; ++s)
          if (r == lane + 32 * s) rmax[s] = mx;
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        int e = 0;
        frexpf(rmax[s], &e);
        rsc[s] = (rmax[s] > 0.f && isfinite(rmax[s])) ? ldexpf(1.f, -e) : 1.f;
      }
      for (int o = 16; o > 0; o >>= 1) afro += __shfl_xor_sync(kFull, afro, o);
      __syncwarp();
      // apply row scales (each lane its rows), identity-pad rows/cols >= n
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        if (r >= NP) continue;
        for (int c = 0; c < NP; ++c) {
          if (r < n && c < n) F(r, c) *= rsc[s];
          else F(r, c) = (r == c) ? 1.f : 0.f;
        }
      }
      __syncwarp();
      // column scales (SPD keeps symmetry: scale columns by the row scale)
      for (int c = lane; c < NP; c += 32) {
        float mx = 0.f;
        for (int r = 0; r < n; ++r) mx = fmaxf(mx, fabsf(F(r, c)));
        int e = 0;
        frexpf(mx, &e);
        float cs = (c < n && mx > 0.f && isfinite(mx)) ? ldexpf(1.f, -e) : 1.f;
        csc[c] = cs;
      }
      __syncwarp();
      if (SPD) {
        for (int c = lane; c < NP; c += 32) {
          // D A D with D = row scales keeps the matrix symmetric
          float d = 1.f;
#pragma unroll
          for (int s = 0; s < MR; ++s)
            if (c == lane + 32 * s) d = rsc[s];
          csc[c] = d;
        }
        __syncwarp();
      }
      for (int r = 0; r < n; ++r)
        for (int c = lane; c < n; c += 32) F(r, c) *= csc[c];
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
        if (SPD) {
          const int ds = k >> 5, dl = k & 31;
          float dv = pan[0][i];
          if (MR > 1 && ds == 1) dv = pan[MR - 1][i];
          const float d = __shfl_sync(kFull, dv, dl);
          if (!(d > 0.f) && info == 0) info = k + 1;
          const float lkk = sqrtf(d > 0.f ? d : 1.f);
          const float ry = 1.f / lkk;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lane + 32 * s;
            if (r == k) pan[s][i] = lkk;
            else if (r > k) pan[s][i] *= ry;
          }
#pragma unroll
          for (int j = i + 1; j < PB; ++j) {
            const int rj = k0 + j;
            float v = pan[0][i];
            if (MR > 1 && (rj >> 5) == 1) v = pan[MR - 1][i];
            const float lj = __shfl_sync(kFull, v, rj & 31);
#pragma unroll
            for (int s = 0; s < MR; ++s)
              if (lane + 32 * s >= rj) pan[s][j] = fmaf(-pan[s][i], lj, pan[s][j]);
          }
          if (lane == 0) ord[k] = k;
        } else {
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
          const int bpos = __reduce_min_sync(kFull, bk == mk ? bp : 0x7fffffff);
          int myslot = -1;
#pragma unroll
          for (int s = 0; s < MR; ++s) myslot = (act[s] && pos[s] == bpos) ? s : myslot;
          const int wl = __ffs(__ballot_sync(kFull, myslot >= 0)) - 1;
          const int wslot = MR > 1 ? __shfl_sync(kFull, myslot, wl) : 0;
          float uw[PB];
#pragma unroll
          for (int j = i; j < PB; ++j) {
            float v = pan[0][j];
            if (MR > 1 && wslot == 1) v = pan[MR - 1][j];
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
          const bool zero = !(uw[i] != 0.f) || !isfinite(uw[i]);
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
      if (!SPD) {
        // U12: the panel's pivot rows on the trailing columns (unit-lower solve)
        for (int j = j1 + lane; j < NP; j += 32) {
          float u[PB];
#pragma unroll
          for (int i = 0; i < PB; ++i) {
            const int pr = ord[k0 + i];
            float acc = F(pr, j);
#pragma unroll
            for (int i2 = 0; i2 < i; ++i2) acc = fmaf(-F(pr, k0 + i2), u[i2], acc);
            u[i] = acc;
            if (i > 0) F(pr, j) = acc;
          }
        }
        __syncwarp();
      }
      // trailing update of the rows still active (SPD: lower triangle rows >= j1)
      if (tc) {
        const int g = lane >> 2, tq = lane & 3;
#pragma unroll
        for (int rt = 0; rt < NP / 16; ++rt) {
          const int ra = rt * 16 + g, rb = ra + 8;
          // skip row tiles with no row to update
          bool upd_a = false, upd_b = false;
          if (SPD) {
            upd_a = ra >= j1;
            upd_b = rb >= j1;
          } else {
            // active after the panel: not yet retired (final position >= j1)
            upd_a = true;
            upd_b = true;
          }
          // L21 fragment (negated): rows ra/rb, panel columns k0 + [2tq, 2tq+1, 2tq+8, 2tq+9]
          unsigned af[4];
          af[0] = pack2(-F(ra, k0 + 2 * tq), -F(ra, k0 + 2 * tq + 1), f16);
          af[1] = pack2(-F(rb, k0 + 2 * tq), -F(rb, k0 + 2 * tq + 1), f16);
          af[2] = pack2(-F(ra, k0 + 2 * tq + 8), -F(ra, k0 + 2 * tq + 9), f16);
          af[3] = pack2(-F(rb, k0 + 2 * tq + 8), -F(rb, k0 + 2 * tq + 9), f16);
          for (int ct = j1 / 8; ct < NP / 8; ++ct) {
            const int c0 = ct * 8 + 2 * tq;
            if (SPD && ct * 8 > rt * 16 + 15) break;  // tile entirely above the diagonal
            // U12 fragment: B[k][n] = U(k0+k, col ct*8+g); SPD: L(col, k0+k)
            unsigned bf[2];
            const int cg = ct * 8 + g;
            if (SPD) {
              bf[0] = pack2(F(cg, k0 + 2 * tq), F(cg, k0 + 2 * tq + 1), f16);
              bf[1] = pack2(F(cg, k0 + 2 * tq + 8), F(cg, k0 + 2 * tq + 9), f16);
            } else {
              bf[0] = pack2(F(ord[k0 + 2 * tq], cg), F(ord[k0 + 2 * tq + 1], cg), f16);
              bf[1] = pack2(F(ord[k0 + 2 * tq + 8], cg), F(ord[k0 + 2 * tq + 9], cg), f16);
            }
            float d[4] = {F(ra, c0), F(ra, c0 + 1), F(rb, c0), F(rb, c0 + 1)};
            mma16816(d, af, bf, f16);
            // store rows that are still being updated
            bool sa = upd_a, sb = upd_b;
            if (!SPD) {
              // a row is updated iff it was active after this panel (its final position is >= j1);
              // positions are known only to the owning lane, so read the active flag via shuffles
              const int la = ra & 31, lb = rb & 31;
              const int va = __shfl_sync(kFull, (int)((ra >> 5) == 0 ? act[0] : act[MR - 1]), la);
              const int vb = __shfl_sync(kFull, (int)((rb >> 5) == 0 ? act[0] : act[MR - 1]), lb);
              sa = va != 0;
              sb = vb != 0;
            }
            if (sa) { F(ra, c0) = d[0]; F(ra, c0 + 1) = d[1]; }
            if (sb) { F(rb, c0) = d[2]; F(rb, c0 + 1) = d[3]; }
          }
        }
      } else {
        // fp32 CUDA-core update, 4 columns at a time
        for (int jc = j1; jc < NP; jc += 4) {
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lane + 32 * s;
            const bool on = SPD ? (r >= j1 && r < NP) : act[s];
            if (!on) continue;
            float4 a4 = F4(r, jc);
            float acc[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
            for (int i = 0; i < PB; ++i) {
              float u[4];
              if (SPD) {
#pragma unroll
                for (int q = 0; q < 4; ++q) u[q] = F(jc + q, k0 + i);
              } else {
                const float4 v = F4(ord[k0 + i], jc);
                u[0] = v.x; u[1] = v.y; u[2] = v.z; u[3] = v.w;
              }
#pragma unroll
              for (int q = 0; q < 4; ++q) acc[q] = fmaf(-pan[s][i], u[q], acc[q]);
            }
            F4(r, jc) = make_float4(acc[0], acc[1], acc[2], acc[3]);
          }
        }
      }
      __syncwarp();
    }
    if (p.info && lane == 0) p.info[m] = info;

    // ---------------------------------------- 3./4. solve and refine in fp64
    // solve(v): v = D_r * rhs (physical rows), returns x = D_c * (U^{-1} L^{-1} P v) into xs
    auto lowsolve = [&](float* v) {
      // forward: y_k at physical row ord[k]; rows retired after k take -L(row,k) y_k
      for (int k = 0; k < NP; ++k) {
        const int pk = ord[k];
        float vk = v[0];
        if (MR > 1 && (pk >> 5) == 1) vk = v[MR - 1];
        float y = __shfl_sync(kFull, vk, pk & 31);
        if (SPD) y = y / F(k, k);  // L is not unit-diagonal for Cholesky
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          const bool after = SPD ? (r > k && r < NP) : (pos[s] > k && r < NP);
          if (after) v[s] = fmaf(-F(r, k), y, v[s]);
          if (SPD && r == k) v[s] = y;
        }
      }
      // backward: x_k = y_k / U(ord[k],k); rows before k take -U(row,k) x_k (SPD: U = L^T)
      for (int k = NP - 1; k >= 0; --k) {
        const int pk = ord[k];
        float vk = v[0];
        if (MR > 1 && (pk >> 5) == 1) vk = v[MR - 1];
        const float x = __shfl_sync(kFull, vk, pk & 31) / F(pk, k);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          if (r == pk) v[s] = x;
          else {
            const bool before = SPD ? (r < k) : (pos[s] < k);
            if (before && r < NP) v[s] = fmaf(-(SPD ? F(k, r) : F(r, k)), x, v[s]);
          }
        }
      }
      // v now holds x by physical row position pk... map to unknown index k: x_k lives at row ord[k]
      __syncwarp();
    };
    // unknowns: for LU the solution component k sits at physical row ord[k] after the back sweep;
    // gather into xs[k] (fp64) scaled by the column scale
    auto gather = [&](const float* v, bool add) {
      for (int k = lane; k < NP; k += 32) {
        const int pk = ord[k];
        (void)pk;
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        if (r >= NP) continue;
        // the row r holds the component of the unknown with position pos (SPD: r)
        const int kk = SPD ? r : pos[s];
        const double xk = (double)v[s] * (double)csc[kk];
        if (kk < n) xs[kk] = add ? xs[kk] + xk : xk;
      }
      __syncwarp();
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
      // r = b - A x, lane r owns rows r, r + 32
      double rr[MR];
      double rn = 0.0, xn = 0.0;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        double acc = bv[s];
        if (r < n) {
          const double* row = Ag + (long long)r * n;
          for (int c = 0; c < n; ++c) acc = fma(-row[c], xs[c], acc);
        }
        rr[s] = (r < n) ? acc : 0.0;
        rn = fma(rr[s], rr[s], rn);
      }
      for (int c = lane; c < n; c += 32) xn = fma(xs[c], xs[c], xn);
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
