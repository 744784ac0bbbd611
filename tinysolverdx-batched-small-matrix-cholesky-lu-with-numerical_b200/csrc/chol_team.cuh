// Batched Cholesky (potrf) fused with the forward and backward substitution
// (posv) — the team kernel described in team.cuh.
//
// Reference semantics (TinySolverDx kernels.hpp:57-87, the default simd backend,
// batched.hpp:121-179, :248-275): lower factor, upper triangle zeroed; info is
// the 1-based index of the first pivot that is not > 0, which is then replaced
// by 1 so the factorization completes; B is overwritten by the solution.
// Per element the chain is the reference's: fused multiply-add for n <= 16,
// separately rounded product and subtraction for n >= 17 (NP <= 16 <=> n <= 16).
#pragma once
#include "team.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS, int TW, int WPC>
struct CholSmem {
  using L = Layout<T, NP, NRHS, TW>;
  static constexpr int STAGE = L::S * L::BUF;
  static constexpr int COL = ((TW > 1) ? 2 : L::S) * NP * int(sizeof(T));
  static constexpr int INFO = (TW > 1) ? 2 * 16 : 0;
  static constexpr int TEAM = ((STAGE + COL + INFO) + 127) / 128 * 128;
  static constexpr int CTA = TEAM * (WPC / TW);
};

template <class T, int NP, int NRHS, int TW, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) chol_team_kernel(SolveArgs<T> p, FastDiv ndiv, int vec) {
  using L = Layout<T, NP, NRHS, TW>;
  using SM = CholSmem<T, NP, NRHS, TW, WPC>;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = L::G, S = L::S, MR = L::MR, MC = L::MC;
  constexpr int VN = V::n;
  constexpr int TPC = WPC / TW, TT = TW * 32;
  constexpr int NA = (TW == 1) ? NP : NP / TW;
  constexpr bool FUSED = NP <= 16;
  extern __shared__ __align__(128) unsigned char smem[];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int team = warp / TW, w = warp % TW, tt = w * 32 + lane;
  const int seg = (G == 32) ? 0 : lane / G;
  const int lsl = lane & (G - 1);
  const int segbase = seg * G;
  unsigned char* stage = smem + team * SM::TEAM;
  T* colb = reinterpret_cast<T*>(stage + SM::STAGE);  // TW == 1: [S][NP]; TW > 1: [2][NP]
  T* sfl = reinterpret_cast<T*>(stage + SM::STAGE + SM::COL);  // TW > 1: [2] {lkk, bad}

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
    if (vec == 16) stage_in<T, 16, L::RS, L::BUF>(stage, reinterpret_cast<const char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    else if (vec == 8) stage_in<T, 8, L::RS, L::BUF>(stage, reinterpret_cast<const char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    else stage_in<T, 4, L::RS, L::BUF>(stage, reinterpret_cast<const char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    cp_async_wait<0>();
    team_sync();

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
    team_sync();

    int info = 0;
    T dinv[MR];
#pragma unroll
    for (int s = 0; s < MR; ++s) dinv[s] = T(1);

#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int OW = L::owner(k), CK = L::slot(k);
      const int ds = k / G, dl = segbase + (k % G);
      T lcol[MR], lkk = T(1);
      bool bad = false;
      T* cb = (TW == 1) ? colb + seg * NP : colb + (k & 1) * NP;
      if (TW == 1 || w == OW) {
        const T d = __shfl_sync(kFull, a[ds][CK], dl);
        bad = !(d > T(0));
        lkk = sqrt_(bad ? T(1) : d);
        const T ry = rcp_(lkk);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          const bool below = r > k && r < NP;
          lcol[s] = T(0);
          if (below) lcol[s] = div_by(a[s][CK], lkk, ry);
          a[s][CK] = below ? lcol[s] : (r == k ? lkk : a[s][CK]);
          if (r < NP) cb[r] = lcol[s];
        }
        if constexpr (TW > 1) {
          if (lane == 0) { sfl[(k & 1) * 2] = lkk; sfl[(k & 1) * 2 + 1] = bad ? T(1) : T(0); }
        }
      }
      if constexpr (TW > 1) {
        named_barrier(1 + team, TT);
        if (w != OW) {
          lkk = sfl[(k & 1) * 2];
          bad = sfl[(k & 1) * 2 + 1] != T(0);
#pragma unroll
          for (int s = 0; s < MR; ++s) lcol[s] = (lsl + G * s < NP) ? cb[lsl + G * s] : T(0);
        }
      } else {
        __syncwarp();
      }
      info = (bad && info == 0) ? k + 1 : info;
      // column k (l_jk for j > k) from shared memory
      T u[NA];
#pragma unroll
      for (int c = 0; c < NA; ++c) u[c] = T(0);
#pragma unroll
      for (int c0 = 0; c0 < NA; c0 += VN) {
        if (L::cmax(c0 + VN - 1) <= k) continue;
        const VT v = *reinterpret_cast<const VT*>(cb + L::col(w, c0));
#pragma unroll
        for (int q = 0; q < VN; ++q) u[c0 + q] = V::get(v, q);
      }
      // trailing update of the lower triangle: k < j <= r
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
#pragma unroll
        for (int c = 0; c < NA; ++c) {
          if (L::cmax(c) <= k) continue;
          const int j = L::col(w, c);
          if (j > k && j <= r && r < NP) a[s][c] = FUSED ? fma_(-lcol[s], u[c], a[s][c]) : sub_mul(a[s][c], lcol[s], u[c]);
        }
      }
      // forward substitution on the right-hand sides this warp owns
      if constexpr (NRHS > 0) {
        const T rk = rcp_(lkk);
        if (lsl == (k % G)) dinv[ds] = rk;
#pragma unroll
        for (int c = NA; c < MC; ++c) {
          const T yk = __shfl_sync(kFull, a[ds][c], dl) * rk;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lsl + G * s;
            const T upd = fma_(-lcol[s], yk, a[s][c]);
            a[s][c] = (r == k) ? yk : ((r > k && r < NP) ? upd : a[s][c]);
          }
        }
      }
      if constexpr (TW == 1) __syncwarp();  // column buffer is rewritten next step
    }

    if (live && w == 0 && lsl == 0 && p.info) p.info[m0 + seg] = info;
    // L -> staging, upper triangle zeroed
    {
      unsigned char* msb = stage + seg * L::BUF;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lsl + G * s;
        if (!(r < NP)) continue;
#pragma unroll
        for (int c0 = 0; c0 < NA; c0 += VN) {
          const int j0 = L::col(w, c0);
          VT v;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(v, q, (j0 + q <= r) ? a[s][c0 + q] : T(0));
          *reinterpret_cast<VT*>(msb + r * L::RS + j0 * int(sizeof(T))) = v;
        }
      }
    }
    team_sync();
    // back substitution L^T x = y (L read back from staging: row k, column r)
    if constexpr (NRHS > 0) {
      const unsigned char* msb = stage + seg * L::BUF;
#pragma unroll
      for (int k = NP - 1; k >= 0; --k) {
        const int ds = k / G, dl = segbase + (k % G);
        T lk[MR];
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          lk[s] = (r < k) ? *reinterpret_cast<const T*>(msb + k * L::RS + r * int(sizeof(T))) : T(0);
        }
#pragma unroll
        for (int c = NA; c < MC; ++c) {
          const T xk = __shfl_sync(kFull, a[ds][c] * dinv[ds], dl);
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lsl + G * s;
            const T upd = fma_(-lk[s], xk, a[s][c]);
            a[s][c] = (r == k) ? xk : ((r < k) ? upd : a[s][c]);
          }
        }
      }
      if (live) {
        const long long bbase = (m0 + seg) * (long long)n * p.ldb + p.b0;
#pragma unroll
        for (int c = NA; c < MC; ++c) {
          const int jb = L::col(w, c) - NP;
          if (jb >= p.nrhs) continue;
#pragma unroll
          for (int s = 0; s < MR; ++s) {
            const int r = lsl + G * s;
            if (r < n) p.B[bbase + (long long)r * p.ldb + jb] = a[s][c];
          }
        }
      }
    }
    if (vec == 16) stage_out<T, 16, L::RS, L::BUF>(stage, reinterpret_cast<char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    else if (vec == 8) stage_out<T, 8, L::RS, L::BUF>(stage, reinterpret_cast<char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    else stage_out<T, 4, L::RS, L::BUF>(stage, reinterpret_cast<char*>(p.A + m0 * nn), cnt * n, n, rc, p.rowdiv, ndiv, tt, TT);
    team_sync();
  }
}

}  // namespace dev
}  // namespace tsdx
