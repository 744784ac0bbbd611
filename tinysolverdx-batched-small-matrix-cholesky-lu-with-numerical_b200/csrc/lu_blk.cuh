// Blocked batched LU with partial pivoting (getrf) fused with the solve (gesv).
//
// One warp per matrix (G lanes per matrix and 32/G matrices per warp for n <= 16).
// The matrix, with its right-hand sides appended as extra columns, lives in
// shared memory; the factorization proceeds in panels of PB columns:
//   1. panel factorization in registers (lane l owns rows l + G*s): pivot search
//      by warp reduction, implicit row swaps, multipliers, rank-1 update of the
//      panel only;
//   2. U12: the panel's pivot rows are brought up to date on the trailing
//      columns by a unit-lower triangular solve (one lane per column);
//   3. trailing update A22 -= L21 U12 for the rows still active, column chunk by
//      column chunk, from shared memory with the multipliers kept in registers.
// Every element still receives exactly the reference's chain of operations
// (TinySolverDx kernels.hpp:91-119: a_ij <- fma(-l_ik, u_kj, a_ij) in increasing k,
// l_ik = a_ik / u_kk correctly rounded, zero pivot => column skipped), so factors,
// pivots and info are bit-identical to the reference; blocking only reorders
// independent element chains. Rows never move: ord[k] records the physical row
// retired at step k, and the output is written in that order, which is where the
// reference's full-row swaps leave each row.
//
// The code is small (the panel body is unrolled PB times, everything else is a
// rolled loop) and every warp of the persistent CTA walks it together.
#pragma once
#include "team.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS>
struct BlkCfg {
  static constexpr int G = NP <= 4 ? 4 : NP <= 8 ? 8 : NP <= 16 ? 16 : 32;  // lanes per matrix
  static constexpr int S = 32 / G;                                          // matrices per warp
  static constexpr int MR = (NP + G - 1) / G;                               // row slots per lane
  static constexpr int PB = NP < 8 ? NP : 8;                                // panel width
  static constexpr int NC = NP + NRHS;                                      // columns incl. B
  static constexpr int CH = 8;                                              // trailing chunk
  static constexpr int NCP = (NC + CH - 1) / CH * CH;                       // row capacity
  // padded row: an odd number of 16-byte units keeps lane-private row accesses conflict-free
  static constexpr int RS = (NCP * int(sizeof(T)) + 31) / 32 * 32 + 16;
  static constexpr int MAT = NP * RS;
  static constexpr int AUX = 2 * NP * 4;  // ord[NP], piv[NP]
  static constexpr int SEGB = (MAT + AUX + 127) / 128 * 128;
  static constexpr int WARPB = S * SEGB;
  static_assert(NP % PB == 0, "panel width divides the padded order");
  static_assert(MR <= 2, "at most two row slots per lane");
};

template <class T, int NP, int NRHS, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) lu_blk_kernel(SolveArgs<T> p, FastDiv ndiv, int vec) {
  using C = BlkCfg<T, NP, NRHS>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = C::G, S = C::S, MR = C::MR, PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS;
  constexpr int VN = V::n;
  constexpr int TS = int(sizeof(T));
  extern __shared__ __align__(128) unsigned char smem[];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int seg = lane / G, lsl = lane & (G - 1), segbase = seg * G;
  const unsigned segmask = (G == 32) ? kFull : (((1u << G) - 1u) << segbase);
  unsigned char* wbase = smem + warp * C::WARPB;
  unsigned char* M = wbase + seg * C::SEGB;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };

  const int n = p.n;
  const long long nn = (long long)n * n;
  const int rc = n * TS / vec;
  const long long per_round = (long long)gridDim.x * WPC * S;

  for (long long base = (long long)blockIdx.x * WPC * S; base < p.batch; base += per_round) {
    __syncthreads();  // the CTA's warps walk the same code together
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
    // identity padding (rows/columns n..NP-1) and the right-hand sides
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

    int pos[MR];
    bool act[MR];
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lsl + G * s;
      act[s] = r < NP;
      pos[s] = r < NP ? r : 0x3fffffff;
    }
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
      unsigned zbits = 0;
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int k = k0 + i;
        K bk = 0;
        int bp = 0x7fffffff;
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const T v = pan[s][i];
          const K key = isnan(v) ? (pos[s] == k ? ~K(0) : K(0)) : key_bits(v) + 1;
          const bool better = act[s] && (key > bk || (key == bk && pos[s] < bp));
          bk = better ? key : bk;
          bp = better ? pos[s] : bp;
        }
        K best;
        const int bpos = seg_argmax(segmask, bk, bp, &best);
        const bool zero = (best == K(1));
        int myslot = -1;
#pragma unroll
        for (int s = 0; s < MR; ++s) myslot = (act[s] && pos[s] == bpos) ? s : myslot;
        const unsigned bal = __ballot_sync(kFull, myslot >= 0);
        const int wl = segbase + __ffs((bal & segmask) >> segbase) - 1;
        int wslot = 0;
        if (MR > 1) wslot = __shfl_sync(kFull, myslot, wl);
        // winner's panel row (columns i..PB-1) to every lane of the segment
        T uw[PB];
#pragma unroll
        for (int j = i; j < PB; ++j) {
          T v = pan[0][j];
          if (MR > 1) v = (wslot == MR - 1) ? pan[MR - 1][j] : v;
          uw[j] = __shfl_sync(kFull, v, wl);
        }
        if (lane == wl) {
          ord[k] = lsl + G * wslot;
          pvs[k] = bpos;
        }
        // retire the winner and replay the reference's swap of positions k and bpos
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const bool win = act[s] && pos[s] == bpos;
          const bool atk = act[s] && !win && pos[s] == k;
          pos[s] = win ? k : (atk ? bpos : pos[s]);
          act[s] = act[s] && !win;
        }
        info = (zero && info == 0) ? k + 1 : info;
        if (zero) {
          zbits |= 1u << i;
        } else {
          const T vpk = uw[i];
          const T ry = rcp_(vpk);
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            if (!act[s]) continue;
            const T l = div_by(pan[s][i], vpk, ry);
            pan[s][i] = l;
#pragma unroll
            for (int j = i + 1; j < PB; ++j) pan[s][j] = fma_(-l, uw[j], pan[s][j]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
        if (r >= NP) continue;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += VN) {
          VT v;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(v, q, pan[s][i0 + q]);
          vat(r, k0 + i0) = v;
        }
      }
      __syncwarp();
      const int j1 = k0 + PB;  // first trailing column
      if (j1 >= NC) continue;
      // ------------------------------- 2. U12: pivot rows on the trailing columns
      for (int j = j1 + lsl; j < NC; j += G) {
        T u[PB];
#pragma unroll
        for (int i = 0; i < PB; ++i) {
          const int pr = ord[k0 + i];
          T acc = at(pr, j);
#pragma unroll
          for (int i2 = 0; i2 < i; ++i2)
            if (!((zbits >> i2) & 1u)) acc = fma_(-at(pr, k0 + i2), u[i2], acc);
          u[i] = acc;
          if (i > 0) at(pr, j) = acc;
        }
      }
      __syncwarp();
      // --------------------------------- 3. trailing update of the active rows
      for (int jc = j1; jc < NC; jc += CH) {
        T acc[MR][CH];
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = act[s] ? lsl + G * s : 0;
#pragma unroll
          for (int c0 = 0; c0 < CH; c0 += VN) {
            const VT v = vat(r, jc + c0);
#pragma unroll
            for (int q = 0; q < VN; ++q) acc[s][c0 + q] = V::get(v, q);
          }
        }
#pragma unroll
        for (int i = 0; i < PB; ++i) {
          if ((zbits >> i) & 1u) continue;
          const int pr = ord[k0 + i];
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
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          if (!act[s]) continue;
          const int r = lsl + G * s;
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

    // ------------------------------------------------- back substitution U x = y
    if constexpr (NRHS > 0) {
      T yv[MR][NRHS], dv[MR];
#pragma unroll
      for (int t = 0; t < MR; ++t) {
        const int i = lsl + G * t;
        const int pr = i < NP ? ord[i] : 0;
        dv[t] = rcp_(at(pr, i < NP ? i : 0));
#pragma unroll
        for (int c = 0; c < NRHS; ++c) yv[t][c] = at(pr, NP + c);
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
            const T u = at(ord[i], k);
#pragma unroll
            for (int c = 0; c < NRHS; ++c) yv[t][c] = fma_(-u, x[c], yv[t][c]);
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
    // ------------------------------------------------------ piv, info, L\U
    if (live) {
      if (p.wf) {
#pragma unroll
        for (int t = 0; t < MR; ++t) {
          const int k = lsl + G * t;
          if (k < n) p.piv[(m0 + seg) * n + k] = pvs[k];
        }
      }
      if (lsl == 0 && p.info) p.info[m0 + seg] = info;
    }
    __syncwarp();
    if (p.wf) {
      char* g = reinterpret_cast<char*>(p.A + m0 * nn);
      const int chunks = cnt * n * rc;
      for (int e = lane; e < chunks; e += 32) {
        const int row = (int)p.rowdiv.div(e), ch = e - row * rc;
        const int mm = (int)ndiv.div(row), r = row - mm * n;
        if (p.status && p.status[m0 + mm] >= 0) continue;
        const unsigned char* mseg = wbase + mm * C::SEGB;
        const int src = reinterpret_cast<const int*>(mseg + C::MAT)[r];
        const unsigned char* sp = mseg + src * RS + ch * vec;
        char* dp = g + (long long)row * n * TS + ch * vec;
        if (vec == 16) *reinterpret_cast<uint4*>(dp) = *reinterpret_cast<const uint4*>(sp);
        else if (vec == 8) *reinterpret_cast<uint2*>(dp) = *reinterpret_cast<const uint2*>(sp);
        else *reinterpret_cast<unsigned*>(dp) = *reinterpret_cast<const unsigned*>(sp);
      }
    }
    __syncwarp();
  }
}

}  // namespace dev
}  // namespace tsdx
