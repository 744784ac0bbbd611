// float64 LU with partial pivoting, one warp per matrix, the trailing update on the
// FP64 tensor cores (mma.sync.m8n8k4.f64), padded orders 32..64.
//
// Layout: the matrix and its right-hand sides (appended as columns, padded to a
// multiple of 8) in shared memory, one padded row per physical row, as in blk.cuh.
// Per panel of 8 columns (k0 = 0, 8, ...):
//   1. pivot steps in registers (lane l holds rows l and l + 32): argmax of |a| by a
//      warp reduction on the high word of the key (exact tie-break only when two
//      lanes share it), the winner's remaining panel row, reciprocal and position
//      published in a shared-memory record, multipliers through that correctly
//      rounded reciprocal, rank-1 update of the panel;
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

// not volatile: the MMA has no effect beyond its outputs, so independent tiles may
// be interleaved by the scheduler
__device__ __forceinline__ void dmma_m8n8k4(double2& c, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c.x), "+d"(c.y)
      : "d"(a), "d"(b));
}


// ---- 1-D bulk copies (TMA, this GPU's own memory, no multicast) on an mbarrier
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity; false if it did not complete within
// kBulkWaitLimit polls (each poll may suspend the warp for a while).
constexpr int kBulkWaitLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  for (int it = 0; it < kBulkWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

template <int NP, int NRHS>
struct TcCfg {
  using B = BlkCfg<double, NP, NRHS, 32>;  // the one-warp row layout of blk.cuh
  static constexpr int RS = B::RS, MAT = B::MAT, MR = B::MR, NC = B::NC, NCP = B::NCP;
  static constexpr int PB = 8;
  static constexpr int NT = NP / 8 - 1;     // most row tiles below a panel
  // ord[NP] (physical row retired at each step), pvs[NP] (pivots), pmap[NP] (position -> row),
  // then the mbarrier of the bulk loads
  static constexpr int OFF_BAR = (MAT + 3 * NP * 4 + 7) / 8 * 8;
  static constexpr int WARPB = (OFF_BAR + 8 + 15) / 16 * 16;
  static_assert(NP % 8 == 0 && NP >= 32 && NP <= 64, "one warp per matrix, two row slots at most");
  static_assert(NCP % 8 == 0, "columns in tiles of 8");
};

// Trailing update of one panel: NTI row tiles of 8 active rows (logical positions
// j1 .. NP - 1 through the position map) against the column tiles from j1 on, the
// right-hand-side tile included. A fragment (lane: tile row fr, k = fq): -l at panel
// columns k0 + fq and k0 + 4 + fq; B fragment (k = fq, column fr): the pivot rows of
// those steps (a zero-pivot step: a = -0, b = +0). NTI == 0: only the right-hand
// sides are left, and they have no active row.
template <int NP, int NRHS, int NTI, bool ZB>
__device__ __forceinline__ void tc_tiles(unsigned char* M, const int* ord, const int* pmap, unsigned zb, int k0,
                                         int lane) {
  if constexpr (NTI > 0) {
    using C = TcCfg<NP, NRHS>;
    constexpr int RS = C::RS, NCP = C::NCP;
    const int fr = lane >> 2, fq = lane & 3, j1 = k0 + 8;
    auto at = [&](int r, int c) -> double& { return *reinterpret_cast<double*>(M + r * RS + c * 8); };
    auto vat = [&](int r, int c) -> double2& { return *reinterpret_cast<double2*>(M + r * RS + c * 8); };
    const bool za = ZB && ((zb >> fq) & 1u), zc = ZB && ((zb >> (4 + fq)) & 1u);
    int prow[NTI];
    double a0[NTI], a1[NTI];
#pragma unroll
    for (int I = 0; I < NTI; ++I) {
      prow[I] = pmap[j1 + 8 * I + fr];
      a0[I] = za ? -0.0 : -at(prow[I], k0 + fq);
      a1[I] = zc ? -0.0 : -at(prow[I], k0 + 4 + fq);
    }
    const int ua = ord[k0 + fq], uc = ord[k0 + 4 + fq];
    for (int J = j1 / 8; J < NCP / 8; ++J) {
      const double b0 = za ? 0.0 : at(ua, 8 * J + fr);
      const double b1 = zc ? 0.0 : at(uc, 8 * J + fr);
      double2 c[NTI];
#pragma unroll
      for (int I = 0; I < NTI; ++I) c[I] = vat(prow[I], 8 * J + 2 * fq);
#pragma unroll
      for (int I = 0; I < NTI; ++I) {
        dmma_m8n8k4(c[I], a0[I], b0);
        dmma_m8n8k4(c[I], a1[I], b1);
      }
#pragma unroll
      for (int I = 0; I < NTI; ++I) vat(prow[I], 8 * J + 2 * fq) = c[I];
    }
  }
}

// U12 (the panel's pivot rows on the trailing columns, one lane per column) and the
// trailing update A22 -= L21 U12 on the tensor cores, for the panel at k0. ZB: the
// panel had a zero-pivot step, which enters both as fma(-(+0), +0, acc) == acc.
template <int NP, int NRHS, bool ZB>
__device__ __forceinline__ void tc_update(unsigned char* M, const int* ord, const int* pmap, unsigned zb, int k0,
                                          int lane) {
  using C = TcCfg<NP, NRHS>;
  using T = double;
  constexpr int PB = C::PB, NC = C::NC, RS = C::RS;
  const int j1 = k0 + PB;
  {
    int prs[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) prs[i] = ord[k0 + i] * RS;
    T l11[PB][PB];
#pragma unroll
    for (int i = 1; i < PB; ++i)
#pragma unroll
      for (int i2 = 0; i2 < i; ++i2)
        l11[i][i2] = (ZB && ((zb >> i2) & 1u)) ? 0.0 : *reinterpret_cast<const T*>(M + prs[i] + (k0 + i2) * 8);
    if (NC - j1 > 32) {
      // two columns per lane, interleaved: two independent chains
      const int jc0 = j1 + lane, jc1 = jc0 + 32;
      const bool two = jc1 < NC;
      T uz0[PB], uz1[PB];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        T* c0 = reinterpret_cast<T*>(M + prs[i] + jc0 * 8);
        T* c1 = reinterpret_cast<T*>(M + prs[i] + (two ? jc1 : jc0) * 8);
        T a0 = *c0, a1 = *c1;
#pragma unroll
        for (int i2 = 0; i2 < i; ++i2) {
          a0 = fma_(-l11[i][i2], uz0[i2], a0);
          a1 = fma_(-l11[i][i2], uz1[i2], a1);
        }
        uz0[i] = (ZB && ((zb >> i) & 1u)) ? 0.0 : a0;
        uz1[i] = (ZB && ((zb >> i) & 1u)) ? 0.0 : a1;
        if (i > 0) {
          *c0 = a0;
          if (two) *c1 = a1;
        }
      }
    } else {
      const int jc = j1 + lane;
      if (jc < NC) {
        T uz[PB];
#pragma unroll
        for (int i = 0; i < PB; ++i) {
          T* cell = reinterpret_cast<T*>(M + prs[i] + jc * 8);
          T acc = *cell;
#pragma unroll
          for (int i2 = 0; i2 < i; ++i2) acc = fma_(-l11[i][i2], uz[i2], acc);
          uz[i] = (ZB && ((zb >> i) & 1u)) ? 0.0 : acc;
          if (i > 0) *cell = acc;
        }
      }
    }
  }
  __syncwarp();
  switch ((NP - j1) / 8) {
    case 7: tc_tiles<NP, NRHS, 7, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 6: tc_tiles<NP, NRHS, 6, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 5: tc_tiles<NP, NRHS, 5, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 4: tc_tiles<NP, NRHS, 4, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 3: tc_tiles<NP, NRHS, 3, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 2: tc_tiles<NP, NRHS, 2, ZB>(M, ord, pmap, zb, k0, lane); break;
    case 1: tc_tiles<NP, NRHS, 1, ZB>(M, ord, pmap, zb, k0, lane); break;
    default: tc_tiles<NP, NRHS, 0, ZB>(M, ord, pmap, zb, k0, lane); break;
  }
  __syncwarp();
}

// Back substitution over physical rows: lane l solves its rows l and l + 32 (at
// positions pos[s]) with the right-hand sides that the factorization left in the
// augmented columns. Step k (from the last position down): the row at position k
// computes x_k = y_k * RN(1/u_kk) and broadcasts it; rows at positions below k take
// y <- fma(-u(row, k), x_k, y) (predicated). A row's y is final after its own step,
// so every row forms its x = y * RN(1/u_kk) once more at the end, the same product.
// These are the operations of a column-oriented back substitution over positions,
// without its per-step selects.
template <int NP, int NRHS>
__device__ __forceinline__ void tc_backsolve(const unsigned char* M, const int* ord, const int (&pos)[TcCfg<NP, NRHS>::MR],
                                             const MatJob<double>& j, int lane) {
  using C = TcCfg<NP, NRHS>;
  constexpr int MR = C::MR, RS = C::RS;
  double y[MR][NRHS], dv[MR];
  const unsigned char* rowp[MR];
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = lane + 32 * s;
    const int rr = r < NP ? r : 0;
    rowp[s] = M + rr * RS;
    dv[s] = rcp_(*reinterpret_cast<const double*>(rowp[s] + (r < NP ? pos[s] : 0) * 8));
#pragma unroll
    for (int c = 0; c < NRHS; ++c) y[s][c] = *reinterpret_cast<const double*>(rowp[s] + (NP + c) * 8);
  }
#pragma unroll 4
  for (int k = NP - 1; k >= 0; --k) {
    const int po = ord[k];
    const bool mine0 = MR == 1 || pos[0] == k;
    const double d = mine0 ? dv[0] : dv[MR - 1];
    double x[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) x[c] = __shfl_sync(kFull, (mine0 ? y[0][c] : y[MR - 1][c]) * d, po & 31);
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const double u = *reinterpret_cast<const double*>(rowp[s] + k * 8);
      const bool below = pos[s] < k;
#pragma unroll
      for (int c = 0; c < NRHS; ++c) fma_if(y[s][c], below, u, x[c]);
    }
  }
  if (j.live && j.B) {
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      if (pos[s] >= j.n) continue;
      double* brow = j.B + (long long)pos[s] * j.ldb + j.b0;
#pragma unroll
      for (int c = 0; c < NRHS; ++c)
        if (c < j.nrhs) brow[c] = y[s][c] * dv[s];
    }
  }
}

// Returns false when the bulk load of the matrix did not complete (the matrix is then
// left unsolved with info = -1).
template <int NP, int NRHS>
__device__ __forceinline__ bool lu_tc_matrix(unsigned char* M, const MatJob<double>& j, int lane, unsigned& par) {
  using C = TcCfg<NP, NRHS>;
  using T = double;
  constexpr int MR = C::MR, PB = C::PB, NC = C::NC, NCP = C::NCP, RS = C::RS, NT = C::NT;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  int* pmap = pvs + NP;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * 8); };
  auto vat = [&](int r, int c) -> double2& { return *reinterpret_cast<double2*>(M + r * RS + c * 8); };

  // ---- stage A and, while it lands, the right-hand sides in registers; identity
  // padding up to NP; the columns that pad the right-hand sides to a whole tile take
  // part in the MMAs and start at zero. Rows whose bytes and start are 16-byte
  // aligned arrive by one bulk copy each (TMA) on the warp's mbarrier, others by
  // per-lane cp.async: issuing 64 cp.async per lane for a 32 KB matrix stalls the
  // warp on the load/store unit for about 13k cycles on B200, the bulk copies take
  // two instructions per lane.
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(M + C::OFF_BAR);
  const int rowb = j.n * 8;
  const bool bulk = (rowb % 16 == 0) && ((reinterpret_cast<unsigned long long>(j.A) & 15) == 0);
  if (bulk) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier smem use before the async writes
    __syncwarp();
    if (lane == 0) mbar_expect_tx(bar, (unsigned)(rowb * j.n));
    __syncwarp();
    for (int r = lane; r < j.n; r += 32)
      bulk_g2s(M + r * RS, reinterpret_cast<const char*>(j.A) + (long long)r * rowb, (unsigned)rowb, bar);
  } else {
    seg_copy_in<T, 32, RS>(M, j.A, j.n, lane);
  }
  T rhs[MR][NRHS > 0 ? NRHS : 1];
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = lane + 32 * s;
    const bool rowok = j.B && r < j.n;
    const T* brow = j.B + (rowok ? (long long)r * j.ldb + j.b0 : 0);
#pragma unroll
    for (int c = 0; c < NRHS; ++c) rhs[s][c] = (rowok && c < j.nrhs) ? brow[c] : T(0);
  }
  if (bulk) {
    const bool ok = mbar_wait_bounded(bar, par);
    if (!__all_sync(kFull, ok)) {
      // the load never completed: report the matrix, wait (bounded) for the copies
      // still in flight to this warp's shared memory, and stop
      if (lane == 0 && j.info) *j.info = -1;
      mbar_wait_bounded(bar, par);
      return false;
    }
    par ^= 1u;
  } else {
    cp_async_wait<0>();
  }
  __syncwarp();
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = lane + 32 * s;
    if (r >= NP) continue;
    for (int c = r >= j.n ? 0 : j.n; c < NP; ++c) at(r, c) = (r == c) ? T(1) : T(0);
#pragma unroll
    for (int c = 0; c < NRHS; ++c) at(r, NP + c) = rhs[s][c];
#pragma unroll
    for (int c = NC; c < NCP; ++c) at(r, c) = 0.0;
  }
  __syncwarp();
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
      const unsigned hi = (unsigned)(bk >> 32);
      const unsigned mhi = __reduce_max_sync(kFull, hi);
      // while the reduction runs: the reciprocal of this lane's candidate (the winner
      // publishes it with its row)
      const T rcand = rcp_((MR > 1 && bs) ? pan[MR - 1][i] : pan[0][i]);
      const unsigned bal = __ballot_sync(kFull, hi == mhi);
      int wl;
      bool zero;
      if (__popc(bal) == 1) {  // one lane holds the largest high word: it wins
        wl = __ffs(bal) - 1;
        zero = false;
      } else {                 // exact tie-break on the full key, then the position
        const unsigned lo = (unsigned)bk;
        const unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
        zero = (mhi == 0u && mlo == 1u);
        const int bx = __reduce_min_sync(kFull, (hi == mhi && lo == mlo) ? bp : 0x7fffffff);
        wl = __ffs(__ballot_sync(kFull, bp == bx)) - 1;
      }
      // the winner's record (80 bytes: panel row, reciprocal, position) in the
      // position-map area, which is free until the panel's map is written
      T* rec = reinterpret_cast<T*>(pmap);
      static_assert(NP * 4 >= 10 * 8, "the record fits the position map");
      if (lane == wl) {
#pragma unroll
        for (int s = 0; s < MR; ++s) {  // stored from the candidate's slot: predicated stores, no selects
          if (bs != s) continue;
#pragma unroll
          for (int jj = i & ~1; jj < PB; jj += 2)
            *reinterpret_cast<double2*>(rec + jj) = make_double2(pan[s][jj], pan[s][jj + 1]);
        }
        rec[8] = rcand;
        reinterpret_cast<int*>(rec + 9)[0] = bp;
        ord[k] = lane + 32 * bs;
        pvs[k] = bp;
      }
      __syncwarp();
      T uw[PB];
#pragma unroll
      for (int jj = i & ~1; jj < PB; jj += 2) {
        const double2 v = *reinterpret_cast<const double2*>(rec + jj);
        uw[jj] = v.x;
        uw[jj + 1] = v.y;
      }
      const T ry = rec[8];
      const int bpos = reinterpret_cast<const int*>(rec + 9)[0];
      __syncwarp();  // all reads done before the next step's record
      // retire the winner and replay the reference's swap of positions k and bpos
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const bool win = pos[s] == bpos;  // retired rows hold positions below k <= bpos
        pos[s] = win ? k : (pos[s] == k ? bpos : pos[s]);
        act[s] = act[s] && !win;
      }
      info = (zero && info == 0) ? k + 1 : info;
      if (zero) {
        zb |= 1u << i;
      } else {
        // l = a / pivot by the shared reciprocal with Markstein's correction (div_by),
        // both rows at once; operands outside its range take the IEEE division on a
        // warp-uniform rare path
        const T vpk = uw[i];
        T l[MR];
        bool slow = false;
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const T a = pan[s][i];
          const T q = __dmul_rn(a, ry);
          const T aq = fabs(q), aa = fabs(a);
          const bool ok = aq >= 0x1p-960 && aq <= 0x1p+960 && aa >= 0x1p-960 && aa <= 0x1p+960;
          const T e = __fma_rn(-vpk, q, a);
          l[s] = ok ? __fma_rn(e, ry, q) : q;  // a zero numerator: q is IEEE's signed zero
          slow = slow || (act[s] && !ok && !(a == 0.0 && q == 0.0));
        }
        if (__any_sync(kFull, slow)) {
#pragma unroll
          for (int s = 0; s < MR; ++s) l[s] = act[s] ? div_by(pan[s][i], vpk, ry) : l[s];
        }
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          if (act[s]) {
            pan[s][i] = l[s];
#pragma unroll
            for (int jj = i + 1; jj < PB; ++jj) pan[s][jj] = fma_(-l[s], uw[jj], pan[s][jj]);
          }
        }
      }
    }
    __syncwarp();  // every lane has read the last record before the position map is written
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
    // ------------------------------- 2. U12 and 3. the trailing update (tensor
    // cores); a panel without a zero pivot (the common case) takes the forms without
    // the zero-pivot selects
    if (zb == 0u) tc_update<NP, NRHS, false>(M, ord, pmap, zb, k0, lane);
    else tc_update<NP, NRHS, true>(M, ord, pmap, zb, k0, lane);
  }

  if constexpr (NRHS > 0) tc_backsolve<NP, NRHS>(M, ord, pos, j, lane);
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
  return true;
}

// Dense batch: a persistent CTA of WPC warps, one matrix per warp per round.
template <int NP, int NRHS, int WPC>
__global__ void __launch_bounds__(WPC * 32, 1) tc_kernel(SolveArgs<double> p) {
  using C = TcCfg<NP, NRHS>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* M = smem + warp * C::WARPB;
  const long long nn = (long long)p.n * p.n;
  const long long step = (long long)gridDim.x * WPC;
  if (lane == 0) mbar_init(reinterpret_cast<unsigned long long*>(M + C::OFF_BAR));
  __syncwarp();
  unsigned par = 0;  // parity of the mbarrier phase the next bulk load completes
  for (long long m = (long long)blockIdx.x * WPC + warp; m < p.batch; m += step) {
    if (p.status && p.status[m] >= 0) continue;  // already solved: nothing to read or write
    // this warp's next matrix heads for L2 while this one is factored
    if (lane == 0 && m + step < p.batch) {
      prefetch_l2(p.A + (m + step) * nn, nn * 8);
      if (p.B) prefetch_l2(p.B + (m + step) * (long long)p.n * p.ldb, (long long)p.n * p.ldb * 8);
    }
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
    if (!lu_tc_matrix<NP, NRHS>(M, j, lane, par)) return;
  }
}

}  // namespace dev
}  // namespace tsdx
