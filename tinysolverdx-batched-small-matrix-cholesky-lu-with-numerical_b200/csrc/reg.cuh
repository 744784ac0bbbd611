// LU with partial pivoting, one warp per matrix with its rows held in registers
// (padded orders 32 and 64).
//
// Lane l owns the physical rows l and l + 32 (MR = NP / 32 row slots). Columns
// [LC, NP) of its rows and the right-hand sides (appended as columns) live in the
// lane's registers; columns [0, LC) live in shared memory (LC = 0: whole rows in
// registers). The shared-memory blocked kernels (blk*.cuh) keep the whole matrix
// in shared memory, which holds 6 float64 matrices of order 64 per SM and spends
// most instructions on shared loads and stores; here the bulk of the trailing
// update is register FMAs on operands broadcast from a small shared buffer.
//
// Factorization in panels of PB = 8 columns, k0 = 0, 8, ...:
//   1. pivot steps on the panel's 8 columns of every row (registers): argmax of
//      |a| over the active rows by a warp reduction on the key's high word, with
//      the exact tie-break only when two lanes share it; the winner publishes its
//      panel row (the panel's L11\U11 block, shared); multipliers through a shared
//      correctly rounded reciprocal; rank-1 update of the panel only;
//   2. U12: the 8 pivot rows publish their register columns to a shared buffer;
//      one lane per 16-byte column group runs the unit-lower triangular solve on
//      them, and on the pivot rows' shared left columns in place; the pivot rows
//      take their finished columns back, and the 8 finished rows' register
//      columns go out to the factor;
//   3. trailing update of the rows still active: register columns in place,
//      shared left columns read-modify-write.
// Panels whose columns sit in shared memory run as a loop; the others are
// unrolled so that every register index is a compile-time constant.
//
// Rows never move: ord[k] is the physical row retired at step k, and the factor
// row k is written from it (as in blk.cuh). Every element receives the
// reference's chain (TinySolverDx kernels.hpp:91-119): a_ij <- fma(-l_ik, u_kj,
// a_ij) in increasing k, l_ik = a_ik / u_kk correctly rounded (div_by), ties to
// the first maximum, NaN never winning off the diagonal position, a zero pivot
// skipping its column. A zero-pivot step enters the delayed updates as
// fma(-(+0), +0, a), which returns a unchanged for every a (signed zeros, Inf and
// NaN included), so the chains stay the reference's. Factors, pivots and info are
// therefore bit-identical to the CPU backends. The forward substitution rides
// along as extra columns; the back substitution is column-oriented with
// reciprocal diagonals (blk.cuh's seg_backsolve order).
#pragma once
#include <utility>

#include "blk.cuh"

namespace tsdx {
namespace dev {

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v / 2); }

template <class F, int... Ps>
__device__ __forceinline__ void for_each_c(F&& f, std::integer_sequence<int, Ps...>) {
  (f(std::integral_constant<int, Ps>{}), ...);
}

template <class T, int NP, int NRHS, int LC>
struct RegCfg {
  static constexpr int TS = int(sizeof(T));
  static constexpr int VN = 16 / TS;        // elements per 16-byte group
  static constexpr int MR = NP / 32;        // row slots per lane
  static constexpr int PB = 8;              // panel width
  static constexpr int NPAN = NP / PB;
  static constexpr int LPAN = LC / PB;      // panels whose columns sit in shared memory
  static constexpr int RC = NP - LC;        // matrix columns in registers
  static constexpr int RW = RC + NRHS;      // register columns per row
  static constexpr int RWP = (RW + VN - 1) / VN * VN;
  static constexpr int NG = RWP / VN;       // 16-byte groups of a register row
  // padded rows: an odd number of 16-byte units keeps row-per-lane accesses conflict-free
  static constexpr int LRS = LC ? ((LC * TS / 16) | 1) * 16 : 0;
  static constexpr int PRS = ((RWP * TS / 16) | 1) * 16;
  static constexpr int OFF_U11 = NP * LRS;             // PB x PB: the pivot rows' panel values
  static constexpr int OFF_PBUF = OFF_U11 + PB * PB * TS;  // PB x RWP: the pivot rows' register columns
  static constexpr int OFF_ORD = OFF_PBUF + PB * PRS;
  static constexpr int OFF_PVS = OFF_ORD + NP * 4;
  static constexpr int MATB = (OFF_PVS + NP * 4 + 127) / 128 * 128;
  static_assert(NP == 32 || NP == 64, "one or two rows per lane");
  static_assert(LC % PB == 0 && LC < NP && (LC == 0 || LC >= PB), "left columns are whole panels");
  static_assert(NG + (LC > PB ? (LC - PB) / VN : 0) <= 32, "one column group per lane in the U12 pass");
};

// Exact warp argmax: the largest key wins, ties go to the smallest position. The
// first reduction runs on the key's high word; when one lane alone holds that
// word, it is the winner and no further reduction is needed. *zero: the winning
// key is 1 (|a| = 0).
__device__ __forceinline__ int warp_argmax(unsigned long long key, int pos, bool* zero) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(kFull, hi);
  const unsigned bal = __ballot_sync(kFull, hi == mhi);
  if (__popc(bal) == 1) {  // then mhi > 0, so the key is not 1
    *zero = false;
    return __shfl_sync(kFull, pos, __ffs(bal) - 1);
  }
  const unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
  *zero = (mhi == 0u && mlo == 1u);
  return __reduce_min_sync(kFull, (hi == mhi && lo == mlo) ? pos : 0x7fffffff);
}
__device__ __forceinline__ int warp_argmax(unsigned key, int pos, bool* zero) {
  const unsigned mk = __reduce_max_sync(kFull, key);
  *zero = (mk == 1u);
  const unsigned bal = __ballot_sync(kFull, key == mk);
  if (__popc(bal) == 1) return __shfl_sync(kFull, pos, __ffs(bal) - 1);
  return __reduce_min_sync(kFull, key == mk ? pos : 0x7fffffff);
}

template <class T, int NP, int NRHS, int LC>
struct RegLU {
  using C = RegCfg<T, NP, NRHS, LC>;
  using K = typename KeyT<T>::U;
  using V = Vec16<T>;
  using VT = typename V::type;
  static constexpr int TS = C::TS, VN = C::VN, MR = C::MR, PB = C::PB, RC = C::RC, RWP = C::RWP, NG = C::NG;
  static constexpr int LRS = C::LRS, PRS = C::PRS, NPAN = C::NPAN, LPAN = C::LPAN;

  unsigned char* M;
  int lane;
  T R[MR][RWP];   // register columns [LC, NP) and the right-hand sides of rows lane + 32 s
  T pan[MR][PB];  // the current panel
  T dg[MR];       // each row's pivot (U diagonal), set when the row is retired
  int pos[MR];    // current position of the row in the reference's row order
  bool act[MR];   // not yet retired
  int info;

  __device__ __forceinline__ VT& vL(int r, int c) const { return *reinterpret_cast<VT*>(M + r * LRS + c * TS); }
  __device__ __forceinline__ T& L(int r, int c) const { return *reinterpret_cast<T*>(M + r * LRS + c * TS); }
  __device__ __forceinline__ VT& vP(int i, int c) const { return *reinterpret_cast<VT*>(M + C::OFF_PBUF + i * PRS + c * TS); }
  __device__ __forceinline__ T& P(int i, int c) const { return *reinterpret_cast<T*>(M + C::OFF_PBUF + i * PRS + c * TS); }
  __device__ __forceinline__ VT& vU(int i, int c) const { return *reinterpret_cast<VT*>(M + C::OFF_U11 + (i * PB + c) * TS); }
  __device__ __forceinline__ int* ord() const { return reinterpret_cast<int*>(M + C::OFF_ORD); }
  __device__ __forceinline__ int* pvs() const { return reinterpret_cast<int*>(M + C::OFF_PVS); }
  __device__ __forceinline__ bool picked(int s, int k0) const { return !act[s] && pos[s] >= k0 && pos[s] < k0 + PB; }
  __device__ static __forceinline__ VT pack(const T* v) {
    VT w;
#pragma unroll
    for (int q = 0; q < VN; ++q) V::set(w, q, v[q]);
    return w;
  }

  // ---- stage the matrix (identity-padded to NP) and the right-hand sides
  __device__ __forceinline__ void load(const MatJob<T>& j) {
    const int n = j.n;
    if constexpr (LC > 0) {
      const int vec = vec_of<T>(j.A, n);
      const char* g = reinterpret_cast<const char*>(j.A);
      const int sh = vec == 16 ? 4 : vec == 8 ? 3 : 2;
      const int cs = ilog2c(LC * TS) - sh;  // log2 of the chunks per row
      for (int e = lane; e < (n << cs); e += 32) {
        const int r = e >> cs, c = (e & ((1 << cs) - 1)) << sh;
        unsigned char* d = M + r * LRS + c;
        const char* s = g + (long long)r * n * TS + c;
        if (vec == 16) cp_async<16>(d, s);
        else if (vec == 8) cp_async<8>(d, s);
        else cp_async<4>(d, s);
      }
      cp_async_commit();
      // padding rows (n > LC: their left columns are all zero)
      for (int e = lane; e < (NP - n) * LC; e += 32) L(n + e / LC, e % LC) = T(0);
    }
    const bool fast = n == NP && (reinterpret_cast<unsigned long long>(j.A) & 15) == 0;
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      const int r = lane + 32 * s;
      const bool real = r < n;
      const T* ar = j.A + (long long)(real ? r : 0) * n + LC;
      if (fast) {
#pragma unroll
        for (int g = 0; g < RC / VN; ++g) {
          const VT v = reinterpret_cast<const VT*>(ar)[g];
#pragma unroll
          for (int q = 0; q < VN; ++q) R[s][g * VN + q] = V::get(v, q);
        }
      } else {
#pragma unroll
        for (int c = 0; c < RC; ++c) R[s][c] = (real && LC + c < n) ? ar[c] : (r == LC + c ? T(1) : T(0));
      }
      const T* br = j.B ? j.B + (long long)(real ? r : 0) * j.ldb + j.b0 : nullptr;
#pragma unroll
      for (int c = 0; c < RWP - RC; ++c) R[s][RC + c] = (br && real && c < NRHS && c < j.nrhs) ? br[c] : T(0);
      pos[s] = r;
      act[s] = true;
      dg[s] = T(0);
    }
    info = 0;
    if constexpr (LC > 0) cp_async_wait<0>();
    __syncwarp();
  }

  // ---- 1. the panel's pivot steps; returns the zero-pivot steps as bits
  __device__ __forceinline__ unsigned pivot_panel(int k0) {
    unsigned zb = 0;
    int* o = ord();
    int* pv = pvs();
#pragma unroll
    for (int i = 0; i < PB; ++i) {
      const int k = k0 + i;
      K bk = 0;
      int bp = 0x7fffffff;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const T v = pan[s][i];
        const K key = isnan(v) ? (pos[s] == k ? ~K(0) : K(0)) : K(key_bits(v) + 1);
        const bool better = act[s] && (key > bk || (key == bk && pos[s] < bp));
        bk = better ? key : bk;
        bp = better ? pos[s] : bp;
      }
      bool zero;
      const int bpos = warp_argmax(bk, bp, &zero);
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const bool win = act[s] && pos[s] == bpos;
        if (win) {
          // the winner's final panel row: multipliers left of i, U beyond
#pragma unroll
          for (int g = 0; g < PB / VN; ++g) vU(i, g * VN) = pack(&pan[s][g * VN]);
          o[k] = lane + 32 * s;
          pv[k] = bpos;
          dg[s] = pan[s][i];
        }
        // retire the winner and replay the reference's swap of positions k and bpos
        const bool atk = act[s] && !win && pos[s] == k;
        pos[s] = win ? k : (atk ? bpos : pos[s]);
        act[s] = act[s] && !win;
      }
      if (zero) {
        info = info ? info : k + 1;
        zb |= 1u << i;
      }
      __syncwarp();
      if (!zero) {
        T u[PB];
#pragma unroll
        for (int g = i / VN; g < PB / VN; ++g) {
          const VT v = vU(i, g * VN);
#pragma unroll
          for (int q = 0; q < VN; ++q) u[g * VN + q] = V::get(v, q);
        }
        const T pk = u[i];
        const T ry = rcp_(pk);
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          if (act[s]) {
            const T l = div_by(pan[s][i], pk, ry);
            pan[s][i] = l;
#pragma unroll
            for (int jj = i + 1; jj < PB; ++jj) pan[s][jj] = fma_(-l, u[jj], pan[s][jj]);
          }
        }
      }
    }
    return zb;
  }

  // ---- 2. U12 of the panel's pivot rows. Lane g < NG takes register group g of the
  // published rows (g >= g0); with LEFT, lanes NG.. take the 16-byte groups of the
  // shared columns [k0 + PB, LC) of the pivot rows, in place.
  template <bool LEFT>
  __device__ __forceinline__ void u12(unsigned zb, int k0, int g0) {
    const int* o = ord();
    const int nl = LEFT ? (LC - k0 - PB) / VN : 0;
    const bool isp = lane >= g0 && lane < NG;
    const bool isl = LEFT && lane >= NG && lane - NG < nl;
    if (!(isp || isl)) return;
    int off[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i)
      off[i] = isp ? C::OFF_PBUF + i * PRS + lane * 16 : o[k0 + i] * LRS + (k0 + PB + (lane - NG) * VN) * TS;
    T u[PB][VN];
#pragma unroll
    for (int i = 0; i < PB; ++i) {
      const VT v = *reinterpret_cast<const VT*>(M + off[i]);
      T acc[VN];
#pragma unroll
      for (int q = 0; q < VN; ++q) acc[q] = V::get(v, q);
      T lr[PB];
#pragma unroll
      for (int g = 0; g < (i + VN - 1) / VN; ++g) {
        const VT w = vU(i, g * VN);
#pragma unroll
        for (int q = 0; q < VN; ++q) lr[g * VN + q] = V::get(w, q);
      }
#pragma unroll
      for (int i2 = 0; i2 < i; ++i2) {
        if ((zb >> i2) & 1u) continue;
#pragma unroll
        for (int q = 0; q < VN; ++q) acc[q] = fma_(-lr[i2], u[i2][q], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < VN; ++q) u[i][q] = acc[q];
      if (i > 0) *reinterpret_cast<VT*>(M + off[i]) = pack(acc);
    }
  }

  // the 8 finished rows' register columns -> factor rows k0 .. k0 + 7, columns [LC, n)
  __device__ __forceinline__ void write_rows(const MatJob<T>& j, int k0) {
    const int n = j.n;
    if (n == NP && (reinterpret_cast<unsigned long long>(j.Aout) & 15) == 0) {
      constexpr int GPR = RC / VN;
      for (int e = lane; e < PB * GPR; e += 32) {
        const int i = e / GPR, g = e % GPR;
        *reinterpret_cast<VT*>(j.Aout + (long long)(k0 + i) * n + LC + g * VN) = vP(i, g * VN);
      }
    } else {
      for (int e = lane; e < PB * RC; e += 32) {
        const int i = e / RC, c = e % RC;
        if (k0 + i < n && LC + c < n) j.Aout[(long long)(k0 + i) * n + LC + c] = P(i, c);
      }
    }
  }

  // ---- 3. trailing update of the active rows' register groups [G1, NG)
  template <int G1>
  __device__ __forceinline__ void trail_regs() {
#pragma unroll
    for (int g = G1; g < NG; ++g) {
      T u[PB][VN];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const VT v = vP(i, g * VN);
#pragma unroll
        for (int q = 0; q < VN; ++q) u[i][q] = V::get(v, q);
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        if (act[s]) {
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            T a = R[s][g * VN + q];
#pragma unroll
            for (int i = 0; i < PB; ++i) a = fma_(-pan[s][i], u[i][q], a);
            R[s][g * VN + q] = a;
          }
        }
      }
    }
  }

  // trailing update of the active rows' shared columns [k0 + PB, LC)
  __device__ __forceinline__ void trail_left(int k0, unsigned zb) {
    const int* o = ord();
    int off[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) off[i] = o[k0 + i] * LRS;
    for (int cg = k0 + PB; cg < LC; cg += VN) {
      T u[PB][VN];
#pragma unroll
      for (int i = 0; i < PB; ++i) {
        const VT v = *reinterpret_cast<const VT*>(M + off[i] + cg * TS);
        const bool z = (zb >> i) & 1u;
#pragma unroll
        for (int q = 0; q < VN; ++q) u[i][q] = z ? T(0) : V::get(v, q);
      }
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        if (act[s]) {
          const int r = lane + 32 * s;
          const VT v = vL(r, cg);
          T a[VN];
#pragma unroll
          for (int q = 0; q < VN; ++q) {
            a[q] = V::get(v, q);
#pragma unroll
            for (int i = 0; i < PB; ++i) a[q] = fma_(-pan[s][i], u[i][q], a[q]);
          }
          vL(r, cg) = pack(a);
        }
      }
    }
  }

  // steps 2 and 3 of a panel; G1: first trailing register group
  template <int G1, bool LEFT>
  __device__ __forceinline__ void panel_tail(const MatJob<T>& j, int k0, unsigned zb) {
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      if (picked(s, k0)) {
        const int i = pos[s] - k0;
#pragma unroll
        for (int g = 0; g < NG; ++g) vP(i, g * VN) = pack(&R[s][g * VN]);
      }
    }
    __syncwarp();
    u12<LEFT>(zb, k0, G1);
    __syncwarp();
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      if (picked(s, k0)) {
        const int i = pos[s] - k0;
#pragma unroll
        for (int g = G1; g < NG; ++g) {
          const VT v = vP(i, g * VN);
#pragma unroll
          for (int q = 0; q < VN; ++q) R[s][g * VN + q] = V::get(v, q);
        }
      }
    }
    if (j.Aout) write_rows(j, k0);
    // zero-pivot steps enter the delayed updates as fma(-(+0), +0, a) == a
#pragma unroll
    for (int s = 0; s < MR; ++s)
#pragma unroll
      for (int i = 0; i < PB; ++i) pan[s][i] = ((zb >> i) & 1u) ? T(0) : pan[s][i];
    if (zb) {
      __syncwarp();
#pragma unroll
      for (int i = 0; i < PB; ++i)
        if ((zb >> i) & 1u)
          for (int g = lane; g < NG; g += 32) vP(i, g * VN) = VT{};
      __syncwarp();
    }
    trail_regs<G1>();
    if constexpr (LEFT) trail_left(k0, zb);
    __syncwarp();
  }

  // column-oriented back substitution step j: x_j from its row's owner, then the
  // rows above it; U(row, j) from getu(slot)
  template <class GU>
  __device__ __forceinline__ void bstep(int j, const T (&ri)[MR], GU getu) {
    constexpr int YC = RC;
    const int owl = ord()[j] & 31;
    T x[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
      T v = R[0][YC + c] * ri[0];
#pragma unroll
      for (int s = 1; s < MR; ++s) v = (pos[s] == j) ? R[s][YC + c] * ri[s] : v;
      x[c] = __shfl_sync(kFull, v, owl);
    }
#pragma unroll
    for (int s = 0; s < MR; ++s) {
      if (pos[s] < j) {
        const T uu = getu(s);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) R[s][YC + c] = fma_(-uu, x[c], R[s][YC + c]);
      } else if (pos[s] == j) {
#pragma unroll
        for (int c = 0; c < NRHS; ++c) R[s][YC + c] = x[c];
      }
    }
  }

  __device__ __forceinline__ void run(const MatJob<T>& j) {
    load(j);
    // panels whose columns sit in shared memory
    for (int p = 0; p < LPAN; ++p) {
      const int k0 = p * PB;
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
#pragma unroll
        for (int g = 0; g < PB / VN; ++g) {
          const VT v = vL(r, k0 + g * VN);
#pragma unroll
          for (int q = 0; q < VN; ++q) pan[s][g * VN + q] = V::get(v, q);
        }
      }
      const unsigned zb = pivot_panel(k0);
#pragma unroll
      for (int s = 0; s < MR; ++s) {
        const int r = lane + 32 * s;
#pragma unroll
        for (int g = 0; g < PB / VN; ++g) vL(r, k0 + g * VN) = pack(&pan[s][g * VN]);
      }
      panel_tail<0, true>(j, k0, zb);
    }
    // panels whose columns sit in registers (unrolled: register indices are constants)
    for_each_c(
        [&](auto PC) {
          constexpr int p = LPAN + decltype(PC)::value;
          constexpr int k0 = p * PB, c0 = k0 - LC, G1 = (c0 + PB) / VN;
#pragma unroll
          for (int s = 0; s < MR; ++s)
#pragma unroll
            for (int i = 0; i < PB; ++i) pan[s][i] = R[s][c0 + i];
          const unsigned zb = pivot_panel(k0);
#pragma unroll
          for (int s = 0; s < MR; ++s)
#pragma unroll
            for (int i = 0; i < PB; ++i) R[s][c0 + i] = pan[s][i];
          panel_tail<G1, false>(j, k0, zb);
        },
        std::make_integer_sequence<int, NPAN - LPAN>{});

    if constexpr (NRHS > 0) {
      T ri[MR];
#pragma unroll
      for (int s = 0; s < MR; ++s) ri[s] = rcp_(dg[s]);
      for_each_c(
          [&](auto JC) {
            constexpr int jj = NP - 1 - decltype(JC)::value;
            bstep(jj, ri, [&](int s) { return R[s][jj - LC]; });
          },
          std::make_integer_sequence<int, RC>{});
      if constexpr (LC > 0) {
        for (int jj = LC - 1; jj >= 0; --jj) bstep(jj, ri, [&](int s) { return L(lane + 32 * s, jj); });
      }
    }
    store(j);
    __syncwarp();
  }

  __device__ __forceinline__ void store(const MatJob<T>& j) {
    const int n = j.n;
    if constexpr (NRHS > 0) {
      if (j.B) {
#pragma unroll
        for (int s = 0; s < MR; ++s) {
          const int r = pos[s];
          if (r < n) {
            T* brow = j.B + (long long)r * j.ldb + j.b0;
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
              if (c < j.nrhs) brow[c] = R[s][RC + c];
          }
        }
      }
    }
    const int* pv = pvs();
    if (j.piv)
      for (int k = lane; k < n; k += 32) j.piv[k] = pv[k];
    if (lane == 0 && j.info) *j.info = info;
    if constexpr (LC > 0) {
      if (j.Aout) {
        // factor columns [0, LC): row k from shared row ord[k]
        const int* o = ord();
        if ((n * TS) % 16 == 0 && (reinterpret_cast<unsigned long long>(j.Aout) & 15) == 0) {
          constexpr int GPR = LC / VN;
          for (int e = lane; e < n * GPR; e += 32) {
            const int k = e / GPR, g = e % GPR;
            *reinterpret_cast<VT*>(j.Aout + (long long)k * n + g * VN) = vL(o[k], g * VN);
          }
        } else {
          for (int e = lane; e < n * LC; e += 32) {
            const int k = e / LC, c = e % LC;
            j.Aout[(long long)k * n + c] = L(o[k], c);
          }
        }
      }
    }
  }
};

// Dense batch: each warp takes matrices m = warp id + i * (warps in the grid).
template <class T, int NP, int NRHS, int LC, int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB) reg_kernel(SolveArgs<T> p) {
  using C = RegCfg<T, NP, NRHS, LC>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long nn = (long long)p.n * p.n;
  RegLU<T, NP, NRHS, LC> w;
  w.M = smem + warp * C::MATB;
  w.lane = lane;
  for (long long m = (long long)blockIdx.x * WPC + warp; m < p.batch; m += (long long)gridDim.x * WPC) {
    if (p.status && p.status[m] >= 0) continue;  // already solved: nothing to read or write
    MatJob<T> j;
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
    w.run(j);
  }
}

}  // namespace dev
}  // namespace tsdx
