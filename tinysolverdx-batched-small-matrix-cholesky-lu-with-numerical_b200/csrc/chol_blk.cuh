// Blocked batched Cholesky (potrf) fused with the solve (posv).
//
// Same execution scheme as lu_blk.cuh: one warp (or one G-lane segment) per
// matrix, the matrix plus its right-hand sides in shared memory, panels of PB
// columns factored in registers, then the trailing lower triangle updated from
// shared memory with the panel multipliers kept in registers.
//
// Reference semantics (TinySolverDx kernels.hpp:57-87, the default simd backend;
// batched.hpp:121-179, :248-275): lower factor with the upper triangle zeroed;
// info = 1-based index of the first pivot that is not > 0, which is replaced by
// 1 so the factorization completes. Each element's chain is the reference's: the
// products of the dot product subtracted in increasing k, fused (one FMA) for
// n <= 16 and separately rounded for n >= 17 (NP <= 16 <=> n <= 16), then a
// correctly rounded division by the diagonal or a square root. The forward
// substitution keeps kernels.hpp:186-193 (fused, then division by l_ii); the
// backward substitution is column-oriented and multiplies by 1/l_ii.
#pragma once
#include "lu_blk.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) chol_blk_kernel(SolveArgs<T> p, FastDiv ndiv, int vec) {
  using C = BlkCfg<T, NP, NRHS>;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = C::G, S = C::S, MR = C::MR, PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS;
  constexpr int VN = V::n;
  constexpr int TS = int(sizeof(T));
  constexpr bool FUSED = NP <= 16;
  extern __shared__ __align__(128) unsigned char smem[];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int seg = lane / G, lsl = lane & (G - 1), segbase = seg * G;
  unsigned char* wbase = smem + warp * C::WARPB;
  unsigned char* M = wbase + seg * C::SEGB;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };
  auto sub = [](T s, T x, T y) -> T { return FUSED ? fma_(-x, y, s) : sub_mul(s, x, y); };

  const int n = p.n;
  const long long nn = (long long)n * n;
  const int rc = n * TS / vec;
  const long long per_round = (long long)gridDim.x * WPC * S;

  for (long long base = (long long)blockIdx.x * WPC * S; base < p.batch; base += per_round) {
    __syncthreads();
    const long long m0 = base + (long long)warp * S;
    if (m0 >= p.batch) continue;
    const int cnt = (int)min((long long)S, p.batch - m0);
    const bool live = seg < cnt && !(p.status && p.status[m0 + seg] >= 0);
    if (!__any_sync(kFull, live)) continue;
    {
      const char* g = reinterpret_cast<const char*>(p.A + m0 * nn);
      if (vec == 16) stage_in<T, 16, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
      else if (vec == 8) stage_in<T, 8, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
      else stage_in<T, 4, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
    }
    cp_async_wait<0>();
    __syncwarp();
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lsl + G * s;
      if (r >= NP) continue;
      const bool full = !live || r >= n;
      for (int c = full ? 0 : n; c < NP; ++c) at(r, c) = (r == c) ? T(1) : T(0);
      if constexpr (NRHS > 0) {
        const long long bb = (m0 + seg) * (long long)n * p.ldb + p.b0 + (long long)r * p.ldb;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) at(r, NP + c) = (live && r < n && c < p.nrhs) ? p.B[bb + c] : T(0);
      }
    }
    __syncwarp();

    int info = 0;
    for (int k0 = 0; k0 < NP; k0 += PB) {
      // ------------------------------------------------ 1. panel in registers
      T pan[MR][PB];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
        const int rr = r < NP ? r : 0;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += VN) {
          const VT v = vat(rr, k0 + i0);
#pragma unroll
          for (int q = 0; q < VN; ++q) pan[s][i0 + q] = V::get(v, q);
        }
      }
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int k = k0 + i;
        const int dl = segbase + (k & (G - 1)), ds = k / G;
        T dv = pan[0][i];
        if (MR > 1) dv = (ds == MR - 1) ? pan[MR - 1][i] : dv;
        const T d = __shfl_sync(kFull, dv, dl);
        const bool bad = !(d > T(0));
        info = (bad && info == 0) ? k + 1 : info;
        const T lkk = sqrt_(bad ? T(1) : d);
        const T ry = rcp_(lkk);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          if (r == k) pan[s][i] = lkk;
          else if (r > k && r < NP) pan[s][i] = div_by(pan[s][i], lkk, ry);
        }
        // multipliers of the panel's own rows k0+j (j > i) for the panel update
#pragma unroll
        for (int j = i + 1; j < PB; ++j) {
          const int rj = k0 + j;
          T v = pan[0][i];
          if (MR > 1) v = ((rj / G) == MR - 1) ? pan[MR - 1][i] : v;
          const T lj = __shfl_sync(kFull, v, segbase + (rj & (G - 1)));
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lsl + G * s;
            if (r >= rj && r < NP) pan[s][j] = sub(pan[s][j], pan[s][i], lj);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
        if (r >= NP || r < k0) continue;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += VN) {
          VT v;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(v, q, pan[s][i0 + q]);
          vat(r, k0 + i0) = v;
        }
      }
      __syncwarp();
      const int j1 = k0 + PB;
      if (j1 >= NC) continue;
      // ------------- 2. forward substitution of the panel rows' right-hand sides
      if constexpr (NRHS > 0) {
        for (int cc = lsl; cc < NRHS; cc += G) {
          const int c = NP + cc;
          T y[PB];
#pragma unroll
          for (int i = 0; i < PB; ++i) {
            const int r = k0 + i;
            T acc = at(r, c);
#pragma unroll
            for (int i2 = 0; i2 < i; ++i2) acc = fma_(-at(r, k0 + i2), y[i2], acc);
            y[i] = div_(acc, at(r, r));
            at(r, c) = y[i];
          }
        }
        __syncwarp();
      }
      // --------------------------- 3. trailing update, rows and columns >= j1
      for (int jc = j1; jc < NC; jc += CH) {
        T acc[MR][CH];
        const bool bcols = jc >= NP;  // a chunk is all-matrix or all-right-hand-side (NP % CH == 0)
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          const int rr = (r >= j1 && r < NP) ? r : 0;
#pragma unroll
          for (int c0 = 0; c0 < CH; c0 += VN) {
            const VT v = vat(rr, jc + c0);
#pragma unroll
            for (int q = 0; q < VN; ++q) acc[s][c0 + q] = V::get(v, q);
          }
        }
        if (!bcols) {
          // a_rj -= sum_i l_ri l_ji over the panel, lower triangle only (j <= r)
#pragma unroll
          for (int c = 0; c < CH; ++c) {
            const int j = jc + c;
#pragma unroll
            for (int i0 = 0; i0 < PB; i0 += VN) {
              const VT v = vat(j, k0 + i0);
#pragma unroll
              for (int q = 0; q < VN; ++q) {
                const T lj = V::get(v, q);
#pragma unroll
                for (int s = 0; s < MR; ++s) {
                  const int r = lsl + G * s;
                  if (j <= r) acc[s][c] = sub(acc[s][c], pan[s][i0 + q], lj);
                }
              }
            }
          }
        } else {
#pragma unroll
          for (int i = 0; i < PB; ++i) {
            const int pr = k0 + i;
#pragma unroll
            for (int c0 = 0; c0 < CH; c0 += VN) {
              const VT v = vat(pr, jc + c0);
#pragma unroll
              for (int q = 0; q < VN; ++q) {
                const T u = V::get(v, q);
#pragma unroll
                for (int s = 0; s < MR; ++s) acc[s][c0 + q] = fma_(-pan[s][i], u, acc[s][c0 + q]);
              }
            }
          }
        }
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          if (r < j1 || r >= NP) continue;
#pragma unroll
          for (int c0 = 0; c0 < CH; c0 += VN) {
            VT v;
#pragma unroll
            for (int q = 0; q < VN; ++q) V::set(v, q, acc[s][c0 + q]);
            vat(r, jc + c0) = v;
          }
        }
      }
      __syncwarp();
    }

    // ---------------------------------------------- back substitution L^T x = y
    if constexpr (NRHS > 0) {
      T yv[MR][NRHS], dv[MR];
#pragma unroll
      for (int t = 0; t < MR; ++t) {
        const int i = lsl + G * t;
        const int ii = i < NP ? i : 0;
        dv[t] = rcp_(at(ii, ii));
#pragma unroll
        for (int c = 0; c < NRHS; ++c) yv[t][c] = at(ii, NP + c);
      }
      for (int k = n - 1; k >= 0; --k) {
        const int ks = k / G, kl = segbase + (k & (G - 1));
        T x[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
          T y = yv[0][c] * dv[0];
          if (MR > 1 && ks == MR - 1) y = yv[MR - 1][c] * dv[MR - 1];
          x[c] = __shfl_sync(kFull, y, kl);
        }
#pragma unroll
        for (int t = 0; t < MR; ++t) {
          const int i = lsl + G * t;
          if (i < k) {
            const T l = at(k, i);
#pragma unroll
            for (int c = 0; c < NRHS; ++c) yv[t][c] = fma_(-l, x[c], yv[t][c]);
          } else if (i == k) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) yv[t][c] = x[c];
          }
        }
      }
      if (live) {
        const long long bb = (m0 + seg) * (long long)n * p.ldb + p.b0;
#pragma unroll
        for (int t = 0; t < MR; ++t) {
          const int i = lsl + G * t;
          if (i >= n) continue;
#pragma unroll
          for (int c = 0; c < NRHS; ++c)
            if (c < p.nrhs) p.B[bb + (long long)i * p.ldb + c] = yv[t][c];
        }
      }
    }
    if (live && lsl == 0 && p.info) p.info[m0 + seg] = info;
    // zero the upper triangle, then copy out
    __syncwarp();
    if (!p.wf) continue;
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lsl + G * s;
      if (r >= NP) continue;
      for (int c = r + 1; c < n; ++c) at(r, c) = T(0);
    }
    __syncwarp();
    if (!p.status) {
      char* g = reinterpret_cast<char*>(p.A + m0 * nn);
      if (vec == 16) stage_out<T, 16, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
      else if (vec == 8) stage_out<T, 8, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
      else stage_out<T, 4, RS, C::SEGB>(wbase, g, cnt * n, n, rc, p.rowdiv, ndiv, lane, 32);
    } else {
      for (int mm = 0; mm < cnt; ++mm) {
        if (p.status[m0 + mm] >= 0) continue;
        char* g = reinterpret_cast<char*>(p.A + (m0 + mm) * nn);
        if (vec == 16) stage_out<T, 16, RS, C::SEGB>(wbase + mm * C::SEGB, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
        else if (vec == 8) stage_out<T, 8, RS, C::SEGB>(wbase + mm * C::SEGB, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
        else stage_out<T, 4, RS, C::SEGB>(wbase + mm * C::SEGB, g, n, n, rc, p.rowdiv, ndiv, lane, 32);
      }
    }
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace tsdx
