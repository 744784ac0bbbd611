// float64 LU with partial pivoting, one warp per matrix, the trailing update on the
// FP64 tensor cores (mma.sync.m8n8k4.f64), padded orders 32..64.
//
// Layout: the matrix and its right-hand sides (appended as columns, padded to a
// multiple of 8) in shared memory, one padded row per physical row, as in blk.cuh.
// Per panel of 8 columns (k0 = 0, 8, ...):
//   1. pivot steps in registers (lane l holds rows l and l + 32): argmax of |a| by a
//      warp reduction on the high word of the key (exact tie-break only when two
//      lanes share it), the winner's remaining panel row broadcast by shuffles,
//      multipliers through a shared correctly rounded reciprocal, rank-1 update of
//      the panel;
//   2. U12: the panel's pivot rows on the trailing columns, one lane per column;
//   3. trailing update A22 -= L21 U12 on 8 x 8 tiles: tile (I, J) covers logical
//      positions j1 + 8I .. j1 + 8I + 7 (gathered through the position -> physical
//      row map, so exactly the rows still active) and columns 8J .. 8J + 7, one
//      m8n8k4 MMA per 4 columns of the panel (two per tile).
//
// Exactness. mma.sync.m8n8k4 with float64 operands accumulates its four products in
// k order as fused multiply-adds, d = fma(a3, b3, fma(a2, b2, fma(a1, b1,
// fma(a0, b0, c)))); this was checked bit for bit against that chain on B200 over
// 4.2 million elements of wide dynamic range (and matches no other order). With
// a = -l_ik and b = u_kj the two MMAs of a tile apply the reference's chain
// a_ij <- fma(-l_ik, u_kj, a_ij) for k = k0 .. k0 + 7 in increasing order
// (TinySolverDx kernels.hpp:111-116), so factors, pivots and info stay
// bit-identical to the CPU backends. A zero-pivot step enters as a = -0, b = +0,
// and fma(-0, +0, c) = c for every c, which is the reference's skipped column.
#pragma once
#include "blk.cuh"

namespace tsdx {
namespace dev {

__device__ __forceinline__ void dmma_m8n8k4(double2& c, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c.x), "+d"(c.y)
               : "d"(a), "d"(b));
}

template <int NP, int NRHS>
struct TcCfg {
  using B = BlkCfg<double, NP, NRHS, 32>;  // the one-warp row layout of blk.cuh
  static constexpr int RS = B::RS, MAT = B::MAT, MR = B::MR, NC = B::NC, NCP = B::NCP;
  static constexpr int PB = 8;
  static constexpr int NT = NP / 8 - 1;     // most row tiles below a panel
  // ord[NP] (physical row retired at each step), pvs[NP] (pivots), pmap[NP] (position -> row)
  static constexpr int WARPB = (MAT + 3 * NP * 4 + 15) / 16 * 16;
  static_assert(NP % 8 == 0 && NP >= 32 && NP <= 64, "one warp per matrix, two row slots at most");
  static_assert(NCP % 8 == 0, "columns in tiles of 8");
};

template <int NP, int NRHS>
__device__ __forceinline__ void lu_tc_matrix(unsigned char* M, const MatJob<double>& j, int lane) {
  using C = TcCfg<NP, NRHS>;
  using T = double;
  constexpr int MR = C::MR, PB = C::PB, NC = C::NC, NCP = C::NCP, RS = C::RS, NT = C::NT;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  int* pmap = pvs + NP;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * 8); };
  auto vat = [&](int r, int c) -> double2& { return *reinterpret_cast<double2*>(M + r * RS + c * 8); };
  Seg g;
  g.lane = lane;
  g.lsl = lane;
  g.segbase = 0;
  g.segmask = kFull;

  seg_load<T, NP, NRHS, 32>(M, j, g);
  // the columns that pad the right-hand sides to a whole tile take part in the MMAs
  if constexpr (NC < NCP) {
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      if (r < NP)
        for (int c = NC; c < NCP; ++c) at(r, c) = 0.0;
    }
  }
  int pos[MR];
  bool act[MR];
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = lane + 32 * s;
    act[s] = r < NP;
    pos[s] = r < NP ? r : 0x3fffffff;
  }
  int info = 0;
  const int fr = lane >> 2, fq = lane & 3;  // MMA fragment row (and B column) and k index

  for (int k0 = 0; k0 < NP; k0 += PB) {
    // ------------------------------------------------ 1. panel in registers
    T pan[MR][PB];
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      const int rr = r < NP ? r : 0;
#pragma unroll
      for (int i0 = 0; i0 < PB; i0 += 2) {
        const double2 v = vat(rr, k0 + i0);
        pan[s][i0] = v.x;
        pan[s][i0 + 1] = v.y;
      }
    }
    unsigned zb = 0;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
      const int k = k0 + i;
      unsigned long long bk = 0;
      int bp = 0x7fffffff, bs = 0;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const T v = pan[s][i];
        const unsigned long long key = isnan(v) ? (pos[s] == k ? ~0ull : 0ull) : key_bits(v) + 1;
        const bool better = act[s] && (key > bk || (key == bk && pos[s] < bp));
        bk = better ? key : bk;
        bp = better ? pos[s] : bp;
        bs = better ? s : bs;
      }
      bool zero;
      int wl;
      const int bpos = warp_argmax_lane(bk, bp, &zero, &wl);
      T uw[PB];  // the winner's panel row, columns i..PB-1
#pragma unroll
      for (int jj = i; jj < PB; ++jj) {
        T v = pan[0][jj];
#pragma unroll
        for (int s = 1; s < MR; ++s) v = (bs == s) ? pan[s][jj] : v;
        uw[jj] = __shfl_sync(kFull, v, wl);
      }
      if (lane == wl) {
        ord[k] = lane + 32 * bs;
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
        zb |= 1u << i;
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
      for (int i0 = 0; i0 < PB; i0 += 2) vat(r, k0 + i0) = make_double2(pan[s][i0], pan[s][i0 + 1]);
      if (act[s]) pmap[pos[s]] = r;
    }
    __syncwarp();
    const int j1 = k0 + PB;
    if (j1 >= NC) continue;
    // ------------------------------- 2. U12: pivot rows on the trailing columns
    for (int jc = j1 + lane; jc < NC; jc += 32) {
      T u[PB];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int pr = ord[k0 + i];
        T acc = at(pr, jc);
#pragma unroll
        for (int i2 = 0; i2 < i; ++i2)
          if (!((zb >> i2) & 1u)) acc = fma_(-at(pr, k0 + i2), u[i2], acc);
        u[i] = acc;
        if (i > 0) at(pr, jc) = acc;
      }
    }
    __syncwarp();
    // --------------------- 3. trailing update on the tensor cores, 8 x 8 tiles
    // A fragment (lane: row fr of the tile, k = fq): -l at panel columns k0 + fq and
    // k0 + 4 + fq; B fragment (k = fq, column fr): the pivot rows of those steps.
    const bool za = (zb >> fq) & 1u, zc = (zb >> (4 + fq)) & 1u;
    int prow[NT];
    T a0[NT], a1[NT];
#pragma unroll
    for (int I = 0; I < NT; ++I) {
      if (j1 + 8 * I < NP) {
        prow[I] = pmap[j1 + 8 * I + fr];
        a0[I] = za ? -0.0 : -at(prow[I], k0 + fq);
        a1[I] = zc ? -0.0 : -at(prow[I], k0 + 4 + fq);
      }
    }
    const int ua = ord[k0 + fq], uc = ord[k0 + 4 + fq];
    for (int J = j1 / 8; J < NCP / 8; ++J) {
      const T b0 = za ? 0.0 : at(ua, 8 * J + fr);
      const T b1 = zc ? 0.0 : at(uc, 8 * J + fr);
#pragma unroll
      for (int I = 0; I < NT; ++I) {
        if (j1 + 8 * I < NP) {
          double2 c = vat(prow[I], 8 * J + 2 * fq);
          dmma_m8n8k4(c, a0[I], b0);
          dmma_m8n8k4(c, a1[I], b1);
          vat(prow[I], 8 * J + 2 * fq) = c;
        }
      }
    }
    __syncwarp();
  }

  if constexpr (NRHS > 0) seg_backsolve<T, NP, NRHS, false, 32>(M, ord, j, g);
  if (j.live) {
    if (j.piv) {
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int k = lane + 32 * s;
        if (k < j.n) j.piv[k] = pvs[k];
      }
    }
    if (lane == 0 && j.info) *j.info = info;
  }
  __syncwarp();
  if (j.live && j.Aout) seg_copy_out<T, 32, RS>(M, j.Aout, j.n, lane, ord);
  __syncwarp();
}

// Dense batch: a persistent CTA of WPC warps, one matrix per warp per round.
template <int NP, int NRHS, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) tc_kernel(SolveArgs<double> p) {
  using C = TcCfg<NP, NRHS>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* M = smem + warp * C::WARPB;
  const long long nn = (long long)p.n * p.n;
  for (long long m = (long long)blockIdx.x * WPC + warp; m < p.batch; m += (long long)gridDim.x * WPC) {
    if (p.status && p.status[m] >= 0) continue;  // already solved: nothing to read or write
    MatJob<double> j;
    j.live = true;
    j.A = p.A + m * nn;
    j.Aout = p.wf ? p.A + m * nn : nullptr;
    j.B = p.B ? p.B + m * (long long)p.n * p.ldb : nullptr;
    j.piv = (p.piv && p.wf) ? p.piv + m * p.n : nullptr;
    j.info = p.info ? p.info + m : nullptr;
    j.n = p.n;
    j.ldb = p.ldb;
    j.b0 = p.b0;
    j.nrhs = p.nrhs;
    lu_tc_matrix<NP, NRHS>(M, j, lane);
  }
}

}  // namespace dev
}  // namespace tsdx
