// LU with partial pivoting, two warps per matrix (orders 33..64).
//
// The one-warp kernel (blk.cuh) is latency-bound at these orders: each lane owns
// two rows, so every pivot step and every trailing-update chunk runs twice per
// lane, and only 6 (fp64) matrices fit an SM. Here a team of two warps owns one
// matrix, thread t (0..63) owns row t:
//   * pivot step: each warp finds its best candidate with redux (as blk.cuh), the
//     candidate's key, position and remaining panel row go to a double-buffered
//     exchange slot in shared memory, one named barrier per step joins the two
//     warps, and both pick the winner with the same comparison (larger key, then
//     smaller position), so the reference's tie-breaking is unchanged;
//   * U12 solve: the trailing columns are dealt to the 64 threads;
//   * trailing update: each thread updates its own row, 8 columns at a time;
//   * back substitution (blk.cuh's, one warp) runs on warp 0 while warp 1 writes
//     the factor and the pivots back.
// Every factor element receives the same chain of operations as in blk.cuh
// (hence as in the reference), so factors, pivots, info and X are bit-identical
// to the one-warp kernel.
#pragma once
#include "blk.cuh"

namespace tsdx {
namespace dev {

template <class T, int NP, int NRHS>
struct Blk2Cfg {
  using B = BlkCfg<T, NP, NRHS, 32>;  // the one-warp layout of the matrix
  static constexpr int RS = B::RS, MAT = B::MAT, PB = B::PB, NC = B::NC, CH = B::CH;
  static constexpr int XSLOT = 16 + PB * int(sizeof(T));  // key (8), position (4), pad, PB values
  static constexpr int XCH = 2 /*buffers*/ * 2 /*warps*/ * XSLOT;
  static constexpr int AUX = 2 * NP * 4;  // ord[NP], pvs[NP]
  static constexpr int TEAMB = (MAT + AUX + XCH + 127) / 128 * 128;
  static_assert(NP > 32 && NP <= 64, "two warps, one row per thread");
};

__device__ __forceinline__ void team_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

template <class T, int NP, int NRHS>
__device__ __forceinline__ void lu2_matrix(unsigned char* M, const MatJob<T>& j, int t, int bar) {
  using C = Blk2Cfg<T, NP, NRHS>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS;
  constexpr int VN = V::n, TS = int(sizeof(T));
  const int lane = t & 31, warp = t >> 5;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  unsigned char* xch = M + C::MAT + C::AUX;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };

  // ---- stage A (rows dealt to the two warps, 16-byte chunks to lanes) and the
  // right-hand sides, identity-pad to NP
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
  const int r = t;
  if (r < NP) {
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

  int pos = r < NP ? r : 0x3fffffff;
  bool act = r < NP;
  const int rr = r < NP ? r : 0;
  int info = 0;
  for (int k0 = 0; k0 < NP; k0 += PB) {
    T pan[PB];
#pragma unroll
    for (int i0 = 0; i0 < PB; i0 += VN) {
      const VT v = vat(rr, k0 + i0);
#pragma unroll
      for (int q = 0; q < VN; ++q) pan[i0 + q] = V::get(v, q);
    }
    unsigned zbits = 0;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
      const int k = k0 + i;
      const T v = pan[i];
      const K key = isnan(v) ? (pos == k ? ~K(0) : K(0)) : key_bits(v) + 1;
      const K bk = act ? key : K(0);
      const int bp = act ? pos : 0x7fffffff;
      K wbest;
      const int wpos = seg_argmax(kFull, bk, bp, &wbest);
      unsigned char* slot = xch + ((k & 1) * 2 + warp) * C::XSLOT;
      if (lane == 0) {
        *reinterpret_cast<K*>(slot) = wbest;
        *reinterpret_cast<int*>(slot + 8) = wpos;
      }
      if (act && pos == wpos) {
        T* sv = reinterpret_cast<T*>(slot + 16);
#pragma unroll
        for (int jj = i; jj < PB; ++jj) sv[jj] = pan[jj];
      }
      team_sync(bar);
      const unsigned char* s0 = xch + ((k & 1) * 2) * C::XSLOT;
      const unsigned char* s1 = s0 + C::XSLOT;
      const K k0v = *reinterpret_cast<const K*>(s0), k1v = *reinterpret_cast<const K*>(s1);
      const int p0 = *reinterpret_cast<const int*>(s0 + 8), p1 = *reinterpret_cast<const int*>(s1 + 8);
      const bool w1 = k1v > k0v || (k1v == k0v && p1 < p0);
      const K best = w1 ? k1v : k0v;
      const int bpos = w1 ? p1 : p0;
      const T* uv = reinterpret_cast<const T*>((w1 ? s1 : s0) + 16);
      T uw[PB];
#pragma unroll
      for (int jj = i; jj < PB; ++jj) uw[jj] = uv[jj];
      const bool win = act && pos == bpos;
      if (win) {
        ord[k] = r;
        pvs[k] = bpos;
      }
      // retire the winner and replay the reference's swap of positions k and bpos
      const bool atk = act && !win && pos == k;
      pos = win ? k : (atk ? bpos : pos);
      act = act && !win;
      const bool zero = (best == K(1));
      info = (zero && info == 0) ? k + 1 : info;
      if (zero) {
        zbits |= 1u << i;
      } else if (act) {
        const T vpk = uw[i];
        const T ry = rcp_(vpk);
        const T l = div_by(pan[i], vpk, ry);
        pan[i] = l;
#pragma unroll
        for (int jj = i + 1; jj < PB; ++jj) pan[jj] = fma_(-l, uw[jj], pan[jj]);
      }
    }
    if (r < NP) {
#pragma unroll
      for (int i0 = 0; i0 < PB; i0 += VN) {
        VT w;
#pragma unroll
        for (int q = 0; q < VN; ++q) V::set(w, q, pan[i0 + q]);
        vat(r, k0 + i0) = w;
      }
    }
    team_sync(bar);
    const int j1 = k0 + PB;
    if (j1 >= NC) continue;
    int ordp[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) ordp[i] = ord[k0 + i];
    // ---- U12: pivot rows on the trailing columns, one column per thread
    for (int jc = j1 + t; jc < NC; jc += 64) {
      T u[PB];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int pr = ordp[i];
        T acc = at(pr, jc);
#pragma unroll
        for (int i2 = 0; i2 < i; ++i2)
          if (!((zbits >> i2) & 1u)) acc = fma_(-at(pr, k0 + i2), u[i2], acc);
        u[i] = acc;
        if (i > 0) at(pr, jc) = acc;
      }
    }
    team_sync(bar);
    // ---- trailing update of the thread's own row (if still active)
    if (act) {
      for (int jc = j1; jc < NC; jc += CH) {
        T acc[CH];
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          const VT v = vat(r, jc + c0);
#pragma unroll
          for (int q = 0; q < VN; ++q) acc[c0 + q] = V::get(v, q);
        }
#pragma unroll
        for (int i = 0; i < PB; ++i) {
          if ((zbits >> i) & 1u) continue;
#pragma unroll
          for (int c0 = 0; c0 < CH; c0 += VN) {
            const VT v = vat(ordp[i], jc + c0);
#pragma unroll
            for (int q = 0; q < VN; ++q) acc[c0 + q] = fma_(-pan[i], V::get(v, q), acc[c0 + q]);
          }
        }
#pragma unroll
        for (int c0 = 0; c0 < CH; c0 += VN) {
          VT w;
#pragma unroll
          for (int q = 0; q < VN; ++q) V::set(w, q, acc[c0 + q]);
          vat(r, jc + c0) = w;
        }
      }
    }
    // the next panel's U12 reads rows other threads update here: its panel barrier orders them
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
  } else if (j.live) {
    if (j.piv)
      for (int k = lane; k < j.n; k += 32) j.piv[k] = pvs[k];
    if (lane == 0 && j.info) *j.info = info;
    if (j.Aout) seg_copy_out<T, 32, RS>(M, j.Aout, j.n, lane, ord);
  }
  team_sync(bar);
}

// Persistent CTA of TPC teams (2 warps each); every round each team takes the next matrix.
template <class T, int NP, int NRHS, int TPC>
__global__ void __launch_bounds__(TPC * 64, 1) blk2_kernel(SolveArgs<T> p) {
  using C = Blk2Cfg<T, NP, NRHS>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int team = threadIdx.x >> 6, t = threadIdx.x & 63;
  unsigned char* M = smem + team * C::TEAMB;
  const long long nn = (long long)p.n * p.n;
  for (long long base = (long long)blockIdx.x * TPC; base < p.batch; base += (long long)gridDim.x * TPC) {
    const long long m = base + team;
    MatJob<T> j;
    j.live = m < p.batch && !(p.status && p.status[m] >= 0);
    // a team with nothing to do (past the batch, or a matrix the status mask marks
    // as already solved) skips the round; its barrier id is private to it
    if (!j.live) continue;
    const long long mm = j.live ? m : 0;
    j.A = p.A + mm * nn;
    j.Aout = p.wf ? p.A + mm * nn : nullptr;
    j.B = p.B ? p.B + mm * (long long)p.n * p.ldb : nullptr;
    j.piv = (p.piv && p.wf) ? p.piv + mm * p.n : nullptr;
    j.info = p.info ? p.info + mm : nullptr;
    j.n = p.n;
    j.ldb = p.ldb;
    j.b0 = p.b0;
    j.nrhs = p.nrhs;
    lu2_matrix<T, NP, NRHS>(M, j, t, 1 + team);
  }
}

}  // namespace dev
}  // namespace tsdx
