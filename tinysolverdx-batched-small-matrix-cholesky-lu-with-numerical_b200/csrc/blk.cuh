// Blocked batched LU with partial pivoting (getrf/gesv) and Cholesky (potrf/posv):
// one G-lane segment per matrix (G = 32 for n > 16; 32/G matrices per warp below),
// the matrix plus its right-hand sides (appended as columns) in shared memory,
// factored in panels of PB columns:
//   1. panel factorization in registers (lane l owns rows l + G*s): LU pivot
//      search by segment reduction with implicit row swaps, or the Cholesky
//      diagonal; multipliers; rank-1 update of the panel only;
//   2. LU: U12, the panel's pivot rows brought up to date on the trailing
//      columns by a unit-lower triangular solve (one lane per column);
//      Cholesky: forward substitution of the panel rows' right-hand sides;
//   3. trailing update A22 -= L21 U12 (Cholesky: the lower triangle, L21 L21^T)
//      for the rows still active, column chunk by column chunk, from shared memory
//      with the panel multipliers kept in registers.
// Every element receives exactly the reference's chain of operations, so factors,
// pivots and info are bit-identical to TinySolverDx's CPU backends:
//   LU (kernels.hpp:91-119): a_ij <- fma(-l_ik, u_kj, a_ij) in increasing k,
//     l_ik = a_ik / u_kk correctly rounded, a zero pivot skips the column; ties go
//     to the first maximum and NaN never wins unless on the diagonal position.
//   Cholesky as the default simd backend compiles kernels.hpp:57-87: the products
//     subtracted in increasing k, fused for n <= 16 and separately rounded for
//     n >= 17 (NP <= 16 <=> n <= 16); a pivot that is not > 0 records info, is
//     replaced by 1 and the factorization completes; the upper triangle is zeroed.
// Rows never move: ord[k] records the physical row retired at step k and the
// factor is written in that order, which is where the reference's full-row swaps
// leave each row. The forward substitution rides along as extra columns (the
// reference's chain, kernels.hpp:184-193 / 214-218); the backward substitution is
// column-oriented with reciprocal diagonals, so X agrees to rounding.
//
// The per-matrix body is a device function over a MatJob (base pointers, sizes),
// shared by the dense-batch kernel below and the uneven-stream kernel.
#pragma once
#include "common.cuh"

namespace tsdx {
namespace dev {

// Hint: bring [p, p + bytes) into L2 (one bulk prefetch; the range is trimmed to
// whole 16-byte units, as the instruction requires).
__device__ __forceinline__ void prefetch_l2(const void* p, long long bytes) {
  const unsigned long long a = reinterpret_cast<unsigned long long>(p);
  const unsigned long long lo = (a + 15) & ~15ull, hi = (a + bytes) & ~15ull;
  if (hi > lo)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

// GO overrides the lanes per matrix (32: one matrix per warp for any NP).
template <class T, int NP, int NRHS, int GO = 0>
struct BlkCfg {
  static constexpr int G = GO ? GO : NP <= 4 ? 4 : NP <= 8 ? 8 : NP <= 16 ? 16 : 32;  // lanes per matrix
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
  static_assert(MR <= 4, "at most four row slots per lane");
};

// One matrix for one segment. Every pointer may be null when the job is not live.
template <class T>
struct MatJob {
  const T* A;   // n x n row-major input
  T* Aout;      // where the factor goes (nullptr: not written)
  T* B;         // n x ldb right-hand sides, columns [b0, b0 + nrhs) solved in place
  int* piv;     // n pivots (LU) or nullptr
  int* info;    // one info word or nullptr
  int n, ldb, b0, nrhs;
  bool live;
};

struct Seg {
  int lane, lsl, segbase;
  unsigned segmask;
};

// Widest copy chunk that keeps every row start aligned.
template <class T> __device__ __forceinline__ int vec_of(const void* p, int n) {
  const unsigned long long a = reinterpret_cast<unsigned long long>(p);
  const int row = n * int(sizeof(T));
  if (row % 16 == 0 && a % 16 == 0) return 16;
  if (row % 8 == 0 && a % 8 == 0) return 8;
  return 4;
}

template <class T, int G, int RS>
__device__ __forceinline__ void seg_copy_in(unsigned char* M, const T* A, int n, int lsl) {
  const int vec = vec_of<T>(A, n);
  const int rc = n * int(sizeof(T)) / vec;
  const char* g = reinterpret_cast<const char*>(A);
  for (int r = 0; r < n; ++r) {
    const char* gr = g + (long long)r * n * int(sizeof(T));
    unsigned char* sr = M + r * RS;
    for (int c = lsl; c < rc; c += G) {
      if (vec == 16) cp_async<16>(sr + c * 16, gr + c * 16);
      else if (vec == 8) cp_async<8>(sr + c * 8, gr + c * 8);
      else cp_async<4>(sr + c * 4, gr + c * 4);
    }
  }
  cp_async_commit();
}

// Copies n rows out of shared memory: output row k <- shared row src[k] (or k).
template <class T, int G, int RS>
__device__ __forceinline__ void seg_copy_out(const unsigned char* M, T* A, int n, int lsl, const int* src) {
  const int vec = vec_of<T>(A, n);
  const int rc = n * int(sizeof(T)) / vec;
  char* g = reinterpret_cast<char*>(A);
  if (vec == 16 && rc <= G && G % rc == 0) {
    // one 16-byte chunk per lane and row, G / rc rows per pass; the passes are
    // independent, so unrolled they keep several loads in flight
    const int rpp = G / rc, c = lsl % rc;
#pragma unroll 4
    for (int k = lsl / rc; k < n; k += rpp) {
      const unsigned char* sr = M + (src ? src[k] : k) * RS;
      *reinterpret_cast<uint4*>(g + (long long)k * n * int(sizeof(T)) + c * 16) =
          *reinterpret_cast<const uint4*>(sr + c * 16);
    }
    return;
  }
  for (int k = 0; k < n; ++k) {
    const unsigned char* sr = M + (src ? src[k] : k) * RS;
    char* gr = g + (long long)k * n * int(sizeof(T));
    for (int c = lsl; c < rc; c += G) {
      if (vec == 16) *reinterpret_cast<uint4*>(gr + c * 16) = *reinterpret_cast<const uint4*>(sr + c * 16);
      else if (vec == 8) *reinterpret_cast<uint2*>(gr + c * 8) = *reinterpret_cast<const uint2*>(sr + c * 8);
      else *reinterpret_cast<unsigned*>(gr + c * 4) = *reinterpret_cast<const unsigned*>(sr + c * 4);
    }
  }
}

// y <- fma(-u, x, y) when p, else y unchanged: one predicated FMA (no select).
__device__ __forceinline__ void fma_if(double& y, bool p, double u, double x) {
  asm("{\n .reg .pred q;\n setp.ne.b32 q, %1, 0;\n @q fma.rn.f64 %0, %2, %3, %0;\n}"
      : "+d"(y)
      : "r"((int)p), "d"(-u), "d"(x));
}
__device__ __forceinline__ void fma_if(float& y, bool p, float u, float x) {
  asm("{\n .reg .pred q;\n setp.ne.b32 q, %1, 0;\n @q fma.rn.f32 %0, %2, %3, %0;\n}"
      : "+f"(y)
      : "r"((int)p), "f"(-u), "f"(x));
}

// Stage the job's matrix (identity-padded to NP) and right-hand sides.
template <class T, int NP, int NRHS, int GO>
__device__ __forceinline__ void seg_load(unsigned char* M, const MatJob<T>& j, const Seg& g) {
  using C = BlkCfg<T, NP, NRHS, GO>;
  constexpr int G = C::G, MR = C::MR, RS = C::RS;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * int(sizeof(T))); };
  if (j.live) seg_copy_in<T, G, RS>(M, j.A, j.n, g.lsl);
  cp_async_wait<0>();
  __syncwarp();
#pragma unroll
  for (int s = 0; s < MR; ++s) {
    const int r = g.lsl + G * s;
    if (r >= NP) continue;
    const bool full = !j.live || r >= j.n;
    for (int c = full ? 0 : j.n; c < NP; ++c) at(r, c) = (r == c) ? T(1) : T(0);
    if constexpr (NRHS > 0) {
      const bool rowok = j.live && j.B && r < j.n;
      const T* brow = rowok ? j.B + (long long)r * j.ldb + j.b0 : nullptr;
#pragma unroll
      for (int c = 0; c < NRHS; ++c) at(r, NP + c) = (rowok && c < j.nrhs) ? brow[c] : T(0);
    }
  }
  __syncwarp();
}

// Column-oriented back substitution with reciprocal diagonals. LU: U(i,k) sits in
// shared row ord[i]; Cholesky: L^T(i,k) = L(k,i).
template <class T, int NP, int NRHS, bool CHOL, int GO>
__device__ __forceinline__ void seg_backsolve(unsigned char* M, const int* ord, const MatJob<T>& j, const Seg& g) {
  using C = BlkCfg<T, NP, NRHS, GO>;
  constexpr int G = C::G, MR = C::MR, RS = C::RS;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * int(sizeof(T))); };
  T yv[MR][NRHS], dv[MR];
  // U(i, k) of this lane's rows at ubase[t] + k * ustride (LU: row ord[i], column k;
  // Cholesky: row k, column i)
  const unsigned char* ubase[MR];
  constexpr int ustride = CHOL ? RS : int(sizeof(T));
#pragma unroll
  for (int t = 0; t < MR; ++t) {
    const int i = g.lsl + G * t;
    const int ii = i < NP ? i : 0;
    const int pr = CHOL ? ii : ord[ii];
    dv[t] = rcp_(at(pr, ii));
    ubase[t] = CHOL ? M + ii * int(sizeof(T)) : M + pr * RS;
#pragma unroll
    for (int c = 0; c < NRHS; ++c) yv[t][c] = at(pr, NP + c);
  }
  // a warp-uniform trip count (segments of one warp may hold different n); the
  // identity-padded positions >= n carry zeros and change nothing. Rows above k take
  // the update as a predicated FMA (U is read for every row; the address is inside
  // the matrix); a row's y is final after its own step, so each row forms its
  // x = y * RN(1/u_ii) once more at the end, the product that was broadcast.
#pragma unroll 4
  for (int k = NP - 1; k >= 0; --k) {
    const int ks = k / G, kl = g.segbase + (k & (G - 1));
    T d = dv[0];
#pragma unroll
    for (int t = 1; t < MR; ++t) d = (ks == t) ? dv[t] : d;
    T x[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
      T y = yv[0][c];
#pragma unroll
      for (int t = 1; t < MR; ++t) y = (ks == t) ? yv[t][c] : y;
      x[c] = __shfl_sync(kFull, y * d, kl);
    }
#pragma unroll
    for (int t = 0; t < MR; ++t) {
      const bool above = g.lsl + G * t < k;
      const T u = *reinterpret_cast<const T*>(ubase[t] + k * ustride);
#pragma unroll
      for (int c = 0; c < NRHS; ++c) fma_if(yv[t][c], above, u, x[c]);
    }
  }
  if (j.live && j.B) {
#pragma unroll
    for (int t = 0; t < MR; ++t) {
      const int i = g.lsl + G * t;
      if (i >= j.n) continue;
      T* brow = j.B + (long long)i * j.ldb + j.b0;
#pragma unroll
      for (int c = 0; c < NRHS; ++c)
        if (c < j.nrhs) brow[c] = yv[t][c] * dv[t];
    }
  }
}

// ------------------------------------------------------------------------- LU
template <class T, int NP, int NRHS, int GO>
__device__ __forceinline__ void lu_matrix(unsigned char* M, const MatJob<T>& j, const Seg& g) {
  using C = BlkCfg<T, NP, NRHS, GO>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = C::G, MR = C::MR, PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS;
  constexpr int VN = V::n, TS = int(sizeof(T));
  const int lane = g.lane, lsl = g.lsl, segbase = g.segbase;
  const unsigned segmask = g.segmask;
  int* ord = reinterpret_cast<int*>(M + C::MAT);
  int* pvs = ord + NP;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };

  seg_load<T, NP, NRHS, GO>(M, j, g);
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
      T uw[PB];  // the winner's panel row, columns i..PB-1
#pragma unroll
      for (int jj = i; jj < PB; ++jj) {
        T v = pan[0][jj];
#pragma unroll
        for (int t = 1; t < MR; ++t) v = (wslot == t) ? pan[t][jj] : v;
        uw[jj] = __shfl_sync(kFull, v, wl);
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
          for (int jj = i + 1; jj < PB; ++jj) pan[s][jj] = fma_(-l, uw[jj], pan[s][jj]);
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
    const int j1 = k0 + PB;
    if (j1 >= NC) continue;
    // ------------------------------- 2. U12: pivot rows on the trailing columns
    for (int jc = j1 + lsl; jc < NC; jc += G) {
      T u[PB];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const int pr = ord[k0 + i];
        T acc = at(pr, jc);
#pragma unroll
        for (int i2 = 0; i2 < i; ++i2)
          if (!((zbits >> i2) & 1u)) acc = fma_(-at(pr, k0 + i2), u[i2], acc);
        u[i] = acc;
        if (i > 0) at(pr, jc) = acc;
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

  if constexpr (NRHS > 0) seg_backsolve<T, NP, NRHS, false, GO>(M, ord, j, g);
  if (j.live) {
    if (j.piv) {
#pragma unroll
      for (int t = 0; t < MR; ++t) {
        const int k = lsl + G * t;
        if (k < j.n) j.piv[k] = pvs[k];
      }
    }
    if (lsl == 0 && j.info) *j.info = info;
  }
  __syncwarp();
  if (j.live && j.Aout) seg_copy_out<T, G, RS>(M, j.Aout, j.n, lsl, ord);
  __syncwarp();
}

// ------------------------------------------------------------------- Cholesky
template <class T, int NP, int NRHS, int GO>
__device__ __forceinline__ void chol_matrix(unsigned char* M, const MatJob<T>& j, const Seg& g) {
  using C = BlkCfg<T, NP, NRHS, GO>;
  using V = Vec16<T>;
  using VT = typename V::type;
  constexpr int G = C::G, MR = C::MR, PB = C::PB, NC = C::NC, CH = C::CH, RS = C::RS;
  constexpr int VN = V::n, TS = int(sizeof(T));
  constexpr bool FUSED = NP <= 16;
  const int lsl = g.lsl, segbase = g.segbase;
  auto at = [&](int r, int c) -> T& { return *reinterpret_cast<T*>(M + r * RS + c * TS); };
  auto vat = [&](int r, int c) -> VT& { return *reinterpret_cast<VT*>(M + r * RS + c * TS); };
  auto sub = [](T s, T x, T y) -> T { return FUSED ? fma_(-x, y, s) : sub_mul(s, x, y); };

  seg_load<T, NP, NRHS, GO>(M, j, g);
  int info = 0;
  for (int k0 = 0; k0 < NP; k0 += PB) {
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
#pragma unroll
      for (int t = 1; t < MR; ++t) dv = (ds == t) ? pan[t][i] : dv;
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
#pragma unroll
      for (int jj = i + 1; jj < PB; ++jj) {
        const int rj = k0 + jj;
        T v = pan[0][i];
#pragma unroll
        for (int t = 1; t < MR; ++t) v = ((rj / G) == t) ? pan[t][i] : v;
        const T lj = __shfl_sync(kFull, v, segbase + (rj & (G - 1)));
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = lsl + G * s;
          if (r >= rj && r < NP) pan[s][jj] = sub(pan[s][jj], pan[s][i], lj);
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
    if constexpr (NRHS > 0) {
      // forward substitution of the panel rows' right-hand sides (fused, then / l_ii)
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
    for (int jc = j1; jc < NC; jc += CH) {
      T acc[MR][CH];
      const bool bcols = jc >= NP;  // NP % CH == 0: a chunk is all-matrix or all-RHS
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
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          const int jcol = jc + c;
#pragma unroll
          for (int i0 = 0; i0 < PB; i0 += VN) {
            const VT v = vat(jcol, k0 + i0);
#pragma unroll
            for (int q = 0; q < VN; ++q) {
              const T lj = V::get(v, q);
#pragma unroll
              for (int s = 0; s < MR; ++s) {
                const int r = lsl + G * s;
                if (jcol <= r) acc[s][c] = sub(acc[s][c], pan[s][i0 + q], lj);
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

  if constexpr (NRHS > 0) seg_backsolve<T, NP, NRHS, true, GO>(M, nullptr, j, g);
  if (j.live && lsl == 0 && j.info) *j.info = info;
  // no early return: every lane of the warp must reach each __syncwarp
  const bool out = j.live && j.Aout;
  __syncwarp();
  if (out) {
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lsl + G * s;
      if (r >= NP) continue;
      for (int c = r + 1; c < j.n; ++c) at(r, c) = T(0);
    }
  }
  __syncwarp();
  if (out) seg_copy_out<T, G, RS>(M, j.Aout, j.n, lsl, nullptr);
  __syncwarp();
}

template <class T, int NP, int NRHS, bool CHOL, int GO = 0>
__device__ __forceinline__ void blk_matrix(unsigned char* M, const MatJob<T>& j, const Seg& g) {
  if constexpr (CHOL) chol_matrix<T, NP, NRHS, GO>(M, j, g);
  else lu_matrix<T, NP, NRHS, GO>(M, j, g);
}

// Dense batch: one persistent CTA of WPC warps per SM slot; every round each
// segment takes the next matrix and the CTA walks the code together, so the
// instruction stream fetched for one warp serves all of them.
template <class T, int NP, int NRHS, int WPC, bool CHOL, int GO = 0>
__global__ void __launch_bounds__(WPC * 32, 1) blk_kernel(SolveArgs<T> p) {
  using C = BlkCfg<T, NP, NRHS, GO>;
  constexpr int G = C::G, S = C::S;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Seg g;
  g.lane = lane;
  g.lsl = lane & (G - 1);
  g.segbase = (lane / G) * G;
  g.segmask = (G == 32) ? kFull : (((1u << G) - 1u) << g.segbase);
  unsigned char* M = smem + warp * C::WARPB + (lane / G) * C::SEGB;
  const long long nn = (long long)p.n * p.n;
  const long long per_round = (long long)gridDim.x * WPC * S;
  // warps own disjoint shared memory, so they run their rounds without a block barrier
  for (long long base = (long long)blockIdx.x * WPC * S; base < p.batch; base += per_round) {
    const long long m = base + (long long)warp * S + lane / G;
    {
      // this warp's next unit heads for L2 while this one is solved
      const long long nxt = base + per_round + (long long)warp * S;
      if (lane == 0 && nxt < p.batch) {
        const long long cnt = (p.batch - nxt) < S ? (p.batch - nxt) : S;
        prefetch_l2(p.A + nxt * nn, cnt * nn * (long long)sizeof(T));
        if (p.B) prefetch_l2(p.B + nxt * (long long)p.n * p.ldb, cnt * (long long)p.n * p.ldb * (long long)sizeof(T));
      }
    }
    MatJob<T> j;
    j.live = m < p.batch && !(p.status && p.status[m] >= 0);
    if (!__any_sync(kFull, j.live)) continue;
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
    blk_matrix<T, NP, NRHS, CHOL, GO>(M, j, g);
  }
}

}  // namespace dev
}  // namespace tsdx
