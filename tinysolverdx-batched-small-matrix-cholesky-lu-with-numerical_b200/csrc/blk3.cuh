// LU with partial pivoting, two warps per matrix with look-ahead (orders 33..64).
//
// Warp 0 (the panel warp) owns the pivoting: it holds the current 8-column panel
// of all rows in registers (two rows per lane, as blk.cuh) and runs the pivot
// steps with intra-warp reductions only. Warp 1 (the update warp) applies each
// panel to the columns beyond the next panel. Per panel p:
//   1. panel warp: pivot steps on panel p, store it, publish the active rows and
//      the zero-pivot bits;                                         barrier S
//   2. both warps: U12 (the panel's pivot rows on the trailing columns, one
//      column per thread);                                          barrier T
//   3. panel warp: apply panel p to panel p + 1's columns (kept in registers)
//      and go straight on to step 1 of panel p + 1, while the update warp
//      applies panel p to every later column.
// So the next panel's pivot chain overlaps the bulk of the trailing update, with
// two named barriers per panel. Every element still receives the updates of the
// panels in increasing order, each as the same chain fma(-l, u, a) over the
// panel's 8 columns in order (blk.cuh), so factors, pivots, info and X are
// bit-identical to the one-warp kernel (and to the reference).
#pragma once
#include "blk2.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS>
struct Blk3Cfg {
  using B = BlkCfg<T, NP, NRHS, 32>;  // the one-warp layout of the matrix
  static constexpr int RS = B::RS, MAT = B::MAT, PB = B::PB, NC = B::NC, CH = B::CH, MR = B::MR;
  static constexpr int NPAN = NP / PB;
  static constexpr int AUX = 2 * NP * 4 + 16;  // ord[NP], pvs[NP], active-row mask, zero-pivot bits
  static constexpr int TEAMB = (MAT + AUX + 127) / 128 * 128;
  static_assert(NP > 32 && NP <= 64 && PB == CH, "two row slots per lane, panel width = chunk width");
};

// SC: the pivot steps of a panel counted in chunk updates. When the update warp has
// R chunks left and R - 1 - SC >= 2, the panel warp takes the last (R - 1 - SC) / 2
// of them, so both warps reach the panel barrier at about the same time.
template <class T, int NP, int NRHS, int SC = 99>
__device__ __forceinline__ void lu3_matrix(unsigned char* M, const MatJob<T>& j, int t, int bar) {
  using C = Blk3Cfg<T, NP, NRHS>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS, MR = C::MR, NPAN = C::NPAN;
  constexpr int VN = V::n, TS = int(sizeof(T));
  const int lane = t & 31, warp = t >> 5;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  unsigned long long* amask = reinterpret_cast<unsigned long long*>(M + C::MAT + 2 * NP * 4);
  unsigned* zpub = reinterpret_cast<unsigned*>(amask + 1);
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };
  // panel k0's update on chunks [jb, je) of the lane's rows (lv: their panel values,
  // ra: still active), the chain of blk.cuh's trailing update
  auto update_chunks = [&](const T (&lv)[MR][PB], const bool (&ra)[MR], const int (&ordp)[PB], unsigned zb,
                           int jb, int je) {
    for (int jc = jb; jc < je; jc += CH) {
      T acc[MR][CH];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int rr = ra[s] ? lane + 32 * s : 0;
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          const VT v = vat(rr, jc + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) acc[s][c0 + q] = V::get(v, q);
        }
      }
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        if ((zb >> i) & 1u) continue;
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          const VT v = vat(ordp[i], jc + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            const T u = V::get(v, q);
#pragma unroll
            for (int s = 0; s < MR; ++s) acc[s][c0 + q] = fma_(-lv[s][i], u, acc[s][c0 + q]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        if (!ra[s]) continue;
        const int r = lane + 32 * s;
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          VT w;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(w, q, acc[s][c0 + q]);
          vat(r, jc + c0) = w;
        }
      }
    }
  };

  // ---- stage A (rows dealt to the two warps) and the right-hand sides
  if (j.live) {
    const int vec = vec_of<T>(j.A, j.n);
    const int rc = j.n * TS / vec;
    const char* g = reinterpret_cast<const char*>(j.A);
    for (int rw = warp; rw < j.n; rw += 2) {
      const char* gr = g + (long long)rw * j.n * TS;
      unsigned char* sr = M + rw * RS;
      for (int c = lane; c < rc; c += 32) {
        if (vec == 16) cp_async<16>(sr + c * 16, gr + c * 16);
        else if (vec == 8) cp_async<8>(sr + c * 8, gr + c * 8);
        else cp_async<4>(sr + c * 4, gr + c * 4);
      }
    }
    cp_async_commit();
  }
  cp_async_wait<0>();
  team_sync(bar);
  if (t < NP) {
    const int r = t;
    const bool full = !j.live || r >= j.n;
    for (int c = full ? 0 : j.n; c < NP; ++c) at(r, c) = (r == c) ? T(1) : T(0);
    if constexpr (NRHS > 0) {
      const bool rowok = j.live && j.B && r < j.n;
      const T* brow = rowok ? j.B + (long long)r * j.ldb + j.b0 : nullptr;
#pragma unroll
      for (int c = 0; c < NRHS; ++c) at(r, NP + c) = (rowok && c < j.nrhs) ? brow[c] : T(0);
    }
  }
  team_sync(bar);

  // panel-warp state (two row slots per lane: rows lane, lane + 32)
  int pos[MR];
  bool act[MR];
  T pan[MR][PB];
  int info = 0;
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = lane + 32 * s;
    act[s] = r < NP;
    pos[s] = r < NP ? r : 0x3fffffff;
  }
  if (warp == 0) {
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int rr = (lane + 32 * s < NP) ? lane + 32 * s : 0;
#pragma unroll
      for (int i0 = 0; i0 < PB; i0 += VN) {
        const VT v = vat(rr, i0);
#pragma unroll
        for (int q = 0; q < VN; ++q) pan[s][i0 + q] = V::get(v, q);
      }
    }
  }

  for (int p = 0; p < NPAN; ++p) {
    const int k0 = p * PB, j1 = k0 + PB;
    if (warp == 0) {
      // ---- 1. pivot steps on the panel (blk.cuh's, one segment of 32 lanes)
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
        const int bpos = seg_argmax(kFull, bk, bp, &best);
        const bool zero = (best == K(1));
        int myslot = -1;
#pragma unroll
        for (int s = 0; s < MR; ++s) myslot = (act[s] && pos[s] == bpos) ? s : myslot;
        const unsigned bal = __ballot_sync(kFull, myslot >= 0);
        const int wl = __ffs(bal) - 1;
        const int wslot = __shfl_sync(kFull, myslot, wl);
        T uw[PB];
#pragma unroll
        for (int jj = i; jj < PB; ++jj) {
          T v = pan[0][jj];
#pragma unroll
          for (int s = 1; s < MR; ++s) v = (wslot == s) ? pan[s][jj] : v;
          uw[jj] = __shfl_sync(kFull, v, wl);
        }
        if (lane == wl) {
          ord[k] = lane + 32 * wslot;
          pvs[k] = bpos;
        }
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
            for (int jj = i + 1; jj < PB; ++jj) pan[s][jj] = fma_(-l, uw[jj], pan[s][jj]);
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        if (r >= NP) continue;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += VN) {
          VT w;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(w, q, pan[s][i0 + q]);
          vat(r, k0 + i0) = w;
        }
      }
      unsigned long long am = 0;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const unsigned b = __ballot_sync(kFull, act[s]);
        am |= (unsigned long long)b << (32 * s);
      }
      if (lane == 0) {
        *amask = am;
        *zpub = zbits;
      }
    }
    team_sync(bar);  // S: panel p, its pivots and the active rows are published
    const unsigned zb = *zpub;
    const unsigned long long am = *amask;
    int ordp[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) ordp[i] = ord[k0 + i];
    // ---- 2. U12: pivot rows on the trailing columns, one column per thread
    for (int jc = j1 + t; jc < NC; jc += 64) {
      T u[PB];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int pr = ordp[i];
        T acc = at(pr, jc);
#pragma unroll
        for (int i2 = 0; i2 < i; ++i2)
          if (!((zb >> i2) & 1u)) acc = fma_(-at(pr, k0 + i2), u[i2], acc);
        u[i] = acc;
        if (i > 0) at(pr, jc) = acc;
      }
    }
    team_sync(bar);  // T: U12 in place
    if (j1 >= NC) continue;
    // chunks beyond the next one: the update warp takes [j1 + CH, jsplit), the
    // panel warp the rest
    const int rem = NC > j1 + CH ? (NC - j1 - CH + CH - 1) / CH : 0;
    const int xtra = rem - 1 - SC >= 2 ? (rem - 1 - SC) / 2 : 0;
    const int jsplit = j1 + CH + (rem - xtra) * CH;
    if (warp == 0) {
      // ---- 3a. the next chunk (panel p + 1, or the right-hand sides after the last
      // panel) for the panel warp's rows, kept in registers for the next pivot steps
      T nxt[MR][PB];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int rr = (lane + 32 * s < NP) ? lane + 32 * s : 0;
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          const VT v = vat(rr, j1 + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) nxt[s][c0 + q] = V::get(v, q);
        }
      }
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        if ((zb >> i) & 1u) continue;
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          const VT v = vat(ordp[i], j1 + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            const T u = V::get(v, q);
#pragma unroll
            for (int s = 0; s < MR; ++s)
              nxt[s][c0 + q] = act[s] ? fma_(-pan[s][i], u, nxt[s][c0 + q]) : nxt[s][c0 + q];
          }
        }
      }
      if (xtra > 0) {
        bool ra[MR];
#pragma unroll
        for (int s = 0; s < MR; ++s) ra[s] = act[s] && lane + 32 * s < NP;
        update_chunks(pan, ra, ordp, zb, jsplit, NC);
      }
      if (p + 1 == NPAN) {
        // the right-hand-side chunk: write it back (the active rows' values changed)
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lane + 32 * s;
          if (r >= NP || !act[s]) continue;
#pragma unroll
          for (int c0 = 0; c0 < CH; c0 += VN) {
            VT w;
#pragma unroll
            for (int q = 0; q < VN; ++q) V::set(w, q, nxt[s][c0 + q]);
            vat(r, j1 + c0) = w;
          }
        }
      } else {
        // the next panel: updated values for the active rows, stored ones for the rest
#pragma unroll
        for (int s = 0; s < MR; ++s)
#pragma unroll
          for (int q = 0; q < PB; ++q) pan[s][q] = nxt[s][q];
      }
    } else {
      // ---- 3b. the update warp: panel p on every column beyond the next chunk
      T lr[MR][PB];
      bool ra[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
        ra[s] = r < NP && ((am >> r) & 1ull);
        const int rr = ra[s] ? r : 0;
#pragma unroll
        for (int i0 = 0; i0 < PB; i0 += VN) {
          const VT v = vat(rr, k0 + i0);
#pragma unroll
          for (int q = 0; q < VN; ++q) lr[s][i0 + q] = V::get(v, q);
        }
      }
      update_chunks(lr, ra, ordp, zb, j1 + CH, jsplit);
    }
    // the next S barrier orders the update warp's writes before the next U12
  }
  team_sync(bar);
  if (warp == 0) {
    if constexpr (NRHS > 0) {
      Seg g0;
      g0.lane = lane;
      g0.lsl = lane;
      g0.segbase = 0;
      g0.segmask = kFull;
      seg_backsolve<T, NP, NRHS, false, 32>(M, ord, j, g0);
    }
    if (j.live && lane == 0 && j.info) *j.info = info;
  } else if (j.live) {
    if (j.piv)
      for (int k = lane; k < j.n; k += 32) j.piv[k] = pvs[k];
    if (j.Aout) seg_copy_out<T, 32, RS>(M, j.Aout, j.n, lane, ord);
  }
  team_sync(bar);
}

template <class T, int NP, int NRHS, int TPC, int SC = 99>
__global__ void __launch_bounds__(TPC * 64, 1) blk3_kernel(SolveArgs<T> p) {
  using C = Blk3Cfg<T, NP, NRHS>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int team = threadIdx.x >> 6, t = threadIdx.x & 63;
  unsigned char* M = smem + team * C::TEAMB;
  const long long nn = (long long)p.n * p.n;
  for (long long base = (long long)blockIdx.x * TPC; base < p.batch; base += (long long)gridDim.x * TPC) {
    const long long m = base + team;
    if (m >= p.batch) continue;  // team-uniform; barrier ids are private to the team
    MatJob<T> j;
    j.live = !(p.status && p.status[m] >= 0);
    if (!j.live) continue;  // already solved (status mask): nothing to read or write
    const long long mm = m;
    j.A = p.A + mm * nn;
    j.Aout = p.wf ? p.A + mm * nn : nullptr;
    j.B = p.B ? p.B + mm * (long long)p.n * p.ldb : nullptr;
    j.piv = (p.piv && p.wf) ? p.piv + mm * p.n : nullptr;
    j.info = p.info ? p.info + mm : nullptr;
    j.n = p.n;
    j.ldb = p.ldb;
    j.b0 = p.b0;
    j.nrhs = p.nrhs;
    lu3_matrix<T, NP, NRHS, SC>(M, j, t, 1 + team);
  }
}

}  // namespace dev
}  // namespace tsdx
