// Batched LU with partial pivoting (getrf) fused with the forward and backward
// substitution (gesv) — the team kernel described in team.cuh.
//
// Reference semantics (TinySolverDx kernels.hpp:91-119, batched.hpp:182-244,
// :259-280): piv[k] is the 0-based position swapped with k; info is the 1-based
// index of the first exactly-zero pivot, after which that column is skipped and
// the factorization completes; A is overwritten by the packed L\U factors and B
// by the solution.
//
// Execution: one persistent CTA of WPC warps per SM slot; every round each team
// of the CTA takes the next matrix and the whole CTA walks the fully unrolled
// code together (a __syncthreads per round), so the instruction stream fetched
// for one warp serves all of them.
#pragma once
#include "team.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS, int TW, int WPC>
struct LuSmem {
  using L = Layout<T, NP, NRHS, TW>;
  static constexpr int STAGE = L::S * L::BUF;
  // per-warp pivot-row buffer, padded so every segment's buffer is 16-byte aligned
  static constexpr int MCP = (L::MC * int(sizeof(T)) + 15) / 16 * 16 / int(sizeof(T));
  static constexpr int UROW = TW * L::S * MCP * int(sizeof(T));
  static constexpr int MULT = (TW > 1) ? 2 * NP * int(sizeof(T)) + 32 : 0;
  static constexpr int TEAM = ((STAGE + UROW + MULT) + 127) / 128 * 128;
  static constexpr int CTA = TEAM * (WPC / TW);
};

template <class T, int NP, int NRHS, int TW, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) lu_team_kernel(SolveArgs<T> p, FastDiv ndiv, int vec) {
  using L = Layout<T, NP, NRHS, TW>;
  using SM = LuSmem<T, NP, NRHS, TW, WPC>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = L::G, S = L::S, MR = L::MR, MC = L::MC;
  constexpr int VN = V::n;
  constexpr int TPC = WPC / TW;                    // teams per CTA
  constexpr int TT = TW * 32;                      // threads per team
  constexpr int NA = (TW == 1) ? NP : NP / TW;     // A-column slots per warp (B slots follow)
  extern __shared__ __align__(128) unsigned char smem[];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int team = warp / TW, w = warp % TW, tt = w * 32 + lane;
  const int seg = (G == 32) ? 0 : lane / G;
  const int lsl = lane & (G - 1);
  const int segbase = seg * G;
  const unsigned segmask = (G == 32) ? kFull : (((1u << G) - 1u) << segbase);
  unsigned char* stage = smem + team * SM::TEAM;
  T* urow = reinterpret_cast<T*>(stage + SM::STAGE) + (w * S + seg) * SM::MCP;
  T* mult = reinterpret_cast<T*>(stage + SM::STAGE + SM::UROW);                                 // [2][NP]
  int* sinfo = reinterpret_cast<int*>(stage + SM::STAGE + SM::UROW + 2 * NP * int(sizeof(T)));  // [2][4]

  auto team_sync = [&]() {
    if constexpr (TW == 1) __syncwarp();
    else named_barrier(1 + team, TT);
  };

  const int n = p.n;
  const long long nn = (long long)n * n;
  const int rc = n * int(sizeof(T)) / vec;
  const long long per_round = (long long)gridDim.x * TPC * S;

  for (long long base = (long long)blockIdx.x * TPC * S; base < p.batch; base += per_round) {
    __syncthreads();  // keep the CTA's warps on the same stretch of code
    const long long m0 = base + (long long)team * S;
    if (m0 >= p.batch) continue;
    const int cnt = (int)min((long long)S, p.batch - m0);
    {
      const char* g = reinterpret_cast<const char*>(p.A + m0 * nn);
      if (vec == 16) stage_in<T, 16, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
      else if (vec == 8) stage_in<T, 8, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
      else stage_in<T, 4, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    }
    cp_async_wait<0>();
    team_sync();

    // ------------------------------------------------------- stage -> registers
    T a[MR][MC];
    const bool live = seg < cnt;
    {
      const unsigned char* ms = stage + seg * L::BUF;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
        const int rr = r < NP ? r : 0;
#pragma unroll
        for (int c0 = 0; c0 < NA; c0 += VN) {
          const int j0 = L::col(w, c0);
          const VT v = *reinterpret_cast<const VT*>(ms + rr * L::RS + j0 * int(sizeof(T)));
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            const int j = j0 + q;
            const bool in = live && r < n && j < n;
            a[s][c0 + q] = in ? V::get(v, q) : (r == j ? T(1) : T(0));
          }
        }
      }
      if constexpr (NRHS > 0) {
        const long long bbase = (m0 + seg) * (long long)n * p.ldb + p.b0;
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
#pragma unroll
          for (int c = NA; c < MC; ++c) {
            const int jb = L::col(w, c) - NP;
            a[s][c] = (live && r < n && jb < p.nrhs) ? p.B[bbase + (long long)r * p.ldb + jb] : T(0);
          }
        }
      }
    }
    team_sync();  // the staging buffer is reused for the output

    // ---------------------------------------------------------- factorization
    int pos[MR], pvv[MR];
    bool act[MR];
    T diag[MR];
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lsl + G * s;
      act[s] = r < NP;
      pos[s] = r < NP ? r : 0x3fffffff;
      pvv[s] = 0;
      diag[s] = T(1);
    }
    int info = 0;

#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int OW = L::owner(k), CK = L::slot(k);
      int bpos = 0, wl = 0, wslot = 0;
      bool zero = false;
      T vpk = T(0);
      T mlt[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) mlt[s] = T(0);
      if (TW == 1 || w == OW) {
        K bk = 0;
        int bp = 0x7fffffff;
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const T v = a[s][CK];
          const K key = isnan(v) ? (pos[s] == k ? ~K(0) : K(0)) : key_bits(v) + 1;
          const bool better = act[s] && (key > bk || (key == bk && pos[s] < bp));
          bk = better ? key : bk;
          bp = better ? pos[s] : bp;
        }
        K best;
        bpos = seg_argmax(segmask, bk, bp, &best);
        zero = (best == K(1));
        int myslot = -1;
#pragma unroll
        for (int s = 0; s < MR; ++s) myslot = (act[s] && pos[s] == bpos) ? s : myslot;
        const unsigned bal = __ballot_sync(kFull, myslot >= 0);
        wl = segbase + __ffs((bal & segmask) >> segbase) - 1;
        if (MR > 1) wslot = __shfl_sync(kFull, myslot, wl);
        T mine = a[0][CK];
        if (MR > 1) mine = (myslot == MR - 1) ? a[MR - 1][CK] : mine;
        vpk = __shfl_sync(kFull, mine, wl);
        const T ry = rcp_(vpk);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const bool doit = act[s] && (myslot != s) && !zero;
          if (doit) {
            mlt[s] = div_by(a[s][CK], vpk, ry);
            a[s][CK] = mlt[s];
          }
        }
        if constexpr (TW > 1) {
          T* mb = mult + (k & 1) * NP;
#pragma unroll
          for (int s = 0; s < MR; ++s)
            if (lsl + G * s < NP) mb[lsl + G * s] = mlt[s];
          if (lane == 0) {
            int* si = sinfo + (k & 1) * 4;
            si[0] = bpos; si[1] = wl; si[2] = wslot; si[3] = zero ? 1 : 0;
          }
        }
      }
      if constexpr (TW > 1) {
        named_barrier(1 + team, TT);
        if (w != OW) {
          const int* si = sinfo + (k & 1) * 4;
          bpos = si[0]; wl = si[1]; wslot = si[2]; zero = si[3] != 0;
          const T* mb = mult + (k & 1) * NP;
#pragma unroll
          for (int s = 0; s < MR; ++s) mlt[s] = (lsl + G * s < NP) ? mb[lsl + G * s] : T(0);
        }
      }
      // retire the pivot row and replay the reference's swap of positions k and bpos
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const bool win = act[s] && pos[s] == bpos;
        const bool atk = act[s] && !win && pos[s] == k;
        if (TW == 1) diag[s] = win ? vpk : diag[s];
        pos[s] = win ? k : (atk ? bpos : pos[s]);
        act[s] = act[s] && !win;
      }
      if (lsl == (k % G)) pvv[k / G] = bpos;
      info = (zero && info == 0) ? k + 1 : info;

      // pivot row, this warp's columns right of k -> shared -> every lane
      __syncwarp();
      if (lane == wl) {
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          if (MR > 1 && s != wslot) continue;
#pragma unroll
          for (int c0 = 0; c0 < MC; c0 += VN) {
            if (L::cmax(c0 + VN - 1 < MC ? c0 + VN - 1 : MC - 1) <= k) continue;
            if (c0 + VN <= MC) {
              VT v;
#pragma unroll
              for (int q = 0; q < VN; ++q) V::set(v, q, a[s][c0 + q]);
              *reinterpret_cast<VT*>(urow + c0) = v;
            } else {
#pragma unroll
              for (int q = 0; q < VN; ++q)
                if (c0 + q < MC) urow[c0 + q] = a[s][c0 + q];
            }
          }
        }
      }
      __syncwarp();
      // rank-1 update of the active rows (the right-hand sides ride along as columns)
#pragma unroll
      for (int c0 = 0; c0 < MC; c0 += VN) {
        if (L::cmax(c0 + VN - 1 < MC ? c0 + VN - 1 : MC - 1) <= k) continue;
        T u[VN];
        if (c0 + VN <= MC) {
          const VT v = *reinterpret_cast<const VT*>(urow + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) u[q] = V::get(v, q);
        } else {
#pragma unroll
          for (int q = 0; q < VN; ++q) u[q] = (c0 + q < MC) ? urow[c0 + q] : T(0);
        }
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const bool rowon = act[s] && !zero;
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            const int c = c0 + q;
            if (c >= MC || L::cmax(c) <= k) continue;
            const bool colon = (L::cmin(c) > k) || (L::col(w, c) > k);
            if (rowon && colon) a[s][c] = fma_(-mlt[s], u[q], a[s][c]);
          }
        }
      }
    }

    // --------------------------------------------------- outputs: piv, info
    if (live && w == 0) {
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int k = lsl + G * s;
        if (k < n) p.piv[(m0 + seg) * n + k] = pvv[s];
      }
      if (lsl == 0 && p.info) p.info[m0 + seg] = info;
    }
    // ------------------------------------------ L\U -> staging, in output order
    {
      unsigned char* msb = stage + seg * L::BUF;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int fp = pos[s];  // final position of this physical row
        if (!(lsl + G * s < NP) || fp >= NP) continue;
#pragma unroll
        for (int c0 = 0; c0 < NA; c0 += VN) {
          const int j0 = L::col(w, c0);
          VT v;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(v, q, a[s][c0 + q]);
          *reinterpret_cast<VT*>(msb + fp * L::RS + j0 * int(sizeof(T))) = v;
        }
      }
    }
    // ------------------------------------------------- back substitution U x = y
    if constexpr (NRHS > 0) {
      if constexpr (TW == 1) {
        T dinv[MR];
#pragma unroll
        for (int s = 0; s < MR; ++s) dinv[s] = rcp_(diag[s]);
#pragma unroll
        for (int k = NP - 1; k >= 0; --k) {
          int own = -1;
#pragma unroll
          for (int s = 0; s < MR; ++s) own = (lsl + G * s < NP && pos[s] == k) ? s : own;
          const unsigned bal = __ballot_sync(kFull, own >= 0);
          const int ol = segbase + __ffs((bal & segmask) >> segbase) - 1;
          T x[NRHS];
#pragma unroll
          for (int r = 0; r < NRHS; ++r) {
            T y = a[0][NP + r] * dinv[0];
            if (MR > 1 && own == MR - 1) y = a[MR - 1][NP + r] * dinv[MR - 1];
            x[r] = __shfl_sync(kFull, y, ol);
          }
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const bool below = (lsl + G * s < NP) && pos[s] < k;
            const bool me = (own == s);
#pragma unroll
            for (int r = 0; r < NRHS; ++r) {
              const T upd = fma_(-a[s][k], x[r], a[s][NP + r]);
              a[s][NP + r] = me ? x[r] : (below ? upd : a[s][NP + r]);
            }
          }
        }
        if (live) {
          const long long bbase = (m0 + seg) * (long long)n * p.ldb + p.b0;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int fp = pos[s];
            if (!(lsl + G * s < NP) || fp >= n) continue;
#pragma unroll
            for (int r = 0; r < NRHS; ++r)
              if (r < p.nrhs) p.B[bbase + (long long)fp * p.ldb + r] = a[s][NP + r];
          }
        }
      } else {
        // TW > 1: U is read back from the staging buffer (row = final position);
        // each warp solves the right-hand sides it owns.
        constexpr int NB = MC - NA;
        named_barrier(1 + team, TT);
        T yv[MR][NB];
#pragma unroll
        for (int s = 0; s < MR; ++s)
#pragma unroll
          for (int c = 0; c < NB; ++c) yv[s][c] = a[s][NA + c];
#pragma unroll
        for (int k = NP - 1; k >= 0; --k) {
          int own = -1;
#pragma unroll
          for (int s = 0; s < MR; ++s) own = (lsl + G * s < NP && pos[s] == k) ? s : own;
          const unsigned bal = __ballot_sync(kFull, own >= 0);
          const int ol = __ffs(bal) - 1;
          const T ukk = *reinterpret_cast<const T*>(stage + k * L::RS + k * int(sizeof(T)));
          const T rinv = rcp_(ukk);
          T x[NB];
#pragma unroll
          for (int c = 0; c < NB; ++c) {
            T y = yv[0][c];
            if (MR > 1 && own == MR - 1) y = yv[MR - 1][c];
            x[c] = __shfl_sync(kFull, y * rinv, ol);
          }
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const bool below = (lsl + G * s < NP) && pos[s] < k;
            const T uik = below ? *reinterpret_cast<const T*>(stage + pos[s] * L::RS + k * int(sizeof(T))) : T(0);
#pragma unroll
            for (int c = 0; c < NB; ++c) {
              const T upd = fma_(-uik, x[c], yv[s][c]);
              yv[s][c] = (own == s) ? x[c] : (below ? upd : yv[s][c]);
            }
          }
        }
        if (live) {
          const long long bbase = m0 * (long long)n * p.ldb + p.b0;
#pragma unroll
          for (int c = 0; c < NB; ++c) {
            const int jb = L::col(w, NA + c) - NP;
            if (jb >= p.nrhs) continue;
#pragma unroll
            for (int s = 0; s < MR; ++s) {
              const int fp = pos[s];
              if ((lsl + G * s < NP) && fp < n) p.B[bbase + (long long)fp * p.ldb + jb] = yv[s][c];
            }
          }
        }
      }
    }
    team_sync();
    {
      char* g = reinterpret_cast<char*>(p.A + m0 * nn);
      if (vec == 16) stage_out<T, 16, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
      else if (vec == 8) stage_out<T, 8, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
      else stage_out<T, 4, L::RS, L::BUF>(stage, g, cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    }
    team_sync();
  }
}

}  // namespace dev
}  // namespace tsdx
