// Learned precision-tier selector: per-matrix features and a 24-64-64-4 MLP with
// its own inference, training (forward + backward) and Adam kernels.
//
// No reference counterpart: TinySolverDx has no mixed-precision path on the GPU.
// The network predicts, per matrix, the cheapest tier {fp16, bf16, fp32, fp64}
// whose refinement (ir.cuh) converges; the refinement's own residual check and
// fp64 fallback make every prediction safe, a wrong one only costs time.
//
// Features (one warp per matrix, one coalesced fp64 pass over A). With
// d_i = |a_ii|, r_i = sum_j |a_ij| (row 1-norm), R_i = r_i - d_i, c_j = sum_i |a_ij|,
// L(x) = log10(max(x, 1e-300)), every feature clipped to [-30, 30]:
//   0 n/64             1 kind (0 SPD, 1 general)   2 L(max d) - L(min d)
//   3 L(max r) - L(min r)    4 L(max c) - L(min c)
//   5 L(max|a|) - L(max d)   6 L(max|a|) - L(min d)  (pivot-growth proxies)
//   7 fraction of rows with d_i > R_i
//   8 min_i (d_i - R_i) / r_i      9 mean_i (d_i - R_i) / r_i   (Gershgorin margins)
//  10 L(max_i (d_i + R_i)) - L(min_i (d_i - R_i))  (Gershgorin bound ratio)
//  11 1 if min_i (d_i - R_i) <= 0                  12 L(||A||_F) - L(max r)
//  13 L(max d) - L(mean d)   14 L(mean d) - L(min d)
//  15 std_i L(d_i)   16 std_i L(r_i)   17 std_j L(c_j)
//  18 max_i (L(r_i) - L(d_i))   19 mean_i (L(r_i) - L(d_i))
//  20 L(||strict lower||_F) - L(||strict upper||_F)
//  21 L(min d) - L(mean_{i != j} |a_ij|)     22 fraction of d_i < 1e-8 max d
//  23 max_j (L(c_j) - L(d_j))
//
// Network (float32): x' = (x - mu) * isd; h1 = relu(W1^T x' + b1) (24 -> 64);
// h2 = relu(W2^T h1 + b2) (64 -> 64); logits = W3^T h2 + b3 (64 -> 4).
// Parameter vector layout: W1[24][64], b1[64], W2[64][64], b2[64], W3[64][4], b3[4].
// Loss: class-weighted softmax cross entropy, sum_s w_{y_s} CE_s / batch.
#pragma once
#include <cuda_runtime.h>

namespace tsdx {
namespace dev {

constexpr int kFeat = 24, kHid = 64, kTiers = 4;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kFeat * kHid, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kTiers, kParams = kOffB3 + kTiers;  // 6020
constexpr int kTrainBlock = 64;   // samples per training block
constexpr int kTrainThreads = 256;

// log10(max(x, 1e-300)) to about 1e-7 absolute: the binary exponent exactly plus a
// single-precision log2 of the mantissa (NaN maps to the clamp, like fmax does).
__device__ __forceinline__ double lg10(double x) {
  if (!(x >= 1e-300)) return -300.0;
  if (x > 1.7976931348623157e308) return 309.0;
  int e = 0;
  const double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
  return ((double)e + (double)__log2f((float)m)) * 0.30102999566398120;
}
__device__ __forceinline__ float clip30(double x) {
  if (!(x == x)) return 0.f;
  return (float)fmin(30.0, fmax(-30.0, x));
}
__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double wmin(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One warp per matrix, one coalesced pass over A in registers: lane c accumulates
// columns c and c + 32, row 1-norms come from per-lane partial sums of 16-row
// chunks folded by a transposing butterfly (lanes 2i and 2i + 1 end with row
// 16 ch + i), then each row's norm is handed to the lane that owns it (row r:
// lane r % 32, slot r / 32, the same lane that holds the diagonal a_rr as part
// of column r).
template <int WPC>
__global__ void __launch_bounds__(WPC * 32) features_kernel(const double* __restrict__ A, int n, long long batch,
                                                            const signed char* kind, int kind_all, float* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  const long long nn = (long long)n * n;
  for (long long m = (long long)blockIdx.x * WPC + warp; m < batch; m += (long long)gridDim.x * WPC) {
    const double* Ag = A + m * nn;
    double csum[2] = {0, 0}, cdg[2] = {0, 0}, cv[4] = {0, 0, 0, 0};
    double amax = 0, lo = 0, up = 0;
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      if (16 * ch < n) {
        double pp[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int r = 16 * ch + j;
          double acc = 0;
          if (r < n) {
            const double* row = Ag + (long long)r * n;
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int c = lane + 32 * s;
              if (c < n) {
                const double v = __ldg(row + c), av = fabs(v), v2 = v * v;
                acc += av;
                csum[s] += av;
                amax = fmax(amax, av);
                if (c < r) lo += v2;
                else if (c > r) up += v2;
                else cdg[s] = av;
              }
            }
          }
          pp[j] = acc;
        }
#pragma unroll
        for (int o = 16, w = 8; w >= 1; o >>= 1, w >>= 1) {
          const bool hi = (lane & o) != 0;
#pragma unroll
          for (int j = 0; j < w; ++j) {
            const double send = hi ? pp[j] : pp[j + w];
            const double keep = hi ? pp[j + w] : pp[j];
            pp[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
          }
        }
        cv[ch] = pp[0] + __shfl_xor_sync(0xffffffffu, pp[0], 1);
      }
    }
    double dmax = 0, dmin = INF, dsum = 0, rmax = 0, rmin = INF, fro = lo + up;
    double dom = 0, gmin = INF, gsum = 0, gup = 0, sld = 0, sld2 = 0, slr = 0, slr2 = 0, rgmax = -INF, rgsum = 0;
    double offs = 0, cmax = 0, cmin = INF, slc = 0, slc2 = 0, cgmax = -INF, gnmin = INF;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double a0 = __shfl_sync(0xffffffffu, cv[2 * s], 2 * (lane & 15));
      const double a1 = __shfl_sync(0xffffffffu, cv[2 * s + 1], 2 * (lane & 15));
      const int r = lane + 32 * s;  // row r and column r
      if (r < n) {
        const double ra = (lane >> 4) ? a1 : a0;
        const double d = cdg[s], R = ra - d;
        fro += d * d;
        dmax = fmax(dmax, d);
        dmin = fmin(dmin, d);
        dsum += d;
        rmax = fmax(rmax, ra);
        rmin = fmin(rmin, ra);
        dom += (d > R) ? 1.0 : 0.0;
        const double g = d - R;
        gmin = fmin(gmin, g);
        gsum += (ra > 0) ? g / ra : 0.0;
        gnmin = fmin(gnmin, (ra > 0) ? g / ra : 0.0);
        gup = fmax(gup, d + R);
        const double ld = lg10(d), lr = lg10(ra);
        sld += ld;
        sld2 += ld * ld;
        slr += lr;
        slr2 += lr * lr;
        rgmax = fmax(rgmax, lr - ld);
        rgsum += lr - ld;
        offs += R;
        const double ca = csum[s], lc = lg10(ca);
        cmax = fmax(cmax, ca);
        cmin = fmin(cmin, ca);
        slc += lc;
        slc2 += lc * lc;
        cgmax = fmax(cgmax, lc - ld);
      }
    }
    dmax = wmax(dmax); dmin = wmin(dmin); dsum = wsum(dsum); rmax = wmax(rmax); rmin = wmin(rmin);
    amax = wmax(amax); fro = wsum(fro); lo = wsum(lo); up = wsum(up); dom = wsum(dom); gmin = wmin(gmin);
    gsum = wsum(gsum); gup = wmax(gup); sld = wsum(sld); sld2 = wsum(sld2); slr = wsum(slr); slr2 = wsum(slr2);
    rgmax = wmax(rgmax); rgsum = wsum(rgsum); offs = wsum(offs); cmax = wmax(cmax); cmin = wmin(cmin);
    slc = wsum(slc); slc2 = wsum(slc2); cgmax = wmax(cgmax); gnmin = wmin(gnmin);
    double tiny = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int r = lane + 32 * s;
      if (r < n && cdg[s] < 1e-8 * dmax) tiny += 1.0;
    }
    tiny = wsum(tiny);
    if (lane == 0) {
      const double fn = (double)n, dmean = dsum / fn;
      float f[kFeat];
      const int kd = kind ? (int)kind[m] : kind_all;
      f[0] = clip30(fn / 64.0);
      f[1] = clip30(kd ? 1.0 : 0.0);
      f[2] = clip30(lg10(dmax) - lg10(dmin));
      f[3] = clip30(lg10(rmax) - lg10(rmin));
      f[4] = clip30(lg10(cmax) - lg10(cmin));
      f[5] = clip30(lg10(amax) - lg10(dmax));
      f[6] = clip30(lg10(amax) - lg10(dmin));
      f[7] = clip30(dom / fn);
      f[8] = clip30(gnmin);
      f[9] = clip30(gsum / fn);
      f[10] = clip30(lg10(gup) - lg10(gmin));
      f[11] = clip30(gmin <= 0 ? 1.0 : 0.0);
      f[12] = clip30(lg10(sqrt(fro)) - lg10(rmax));
      f[13] = clip30(lg10(dmax) - lg10(dmean));
      f[14] = clip30(lg10(dmean) - lg10(dmin));
      f[15] = clip30(sqrt(fmax(0.0, sld2 / fn - (sld / fn) * (sld / fn))));
      f[16] = clip30(sqrt(fmax(0.0, slr2 / fn - (slr / fn) * (slr / fn))));
      f[17] = clip30(sqrt(fmax(0.0, slc2 / fn - (slc / fn) * (slc / fn))));
      f[18] = clip30(rgmax);
      f[19] = clip30(rgsum / fn);
      f[20] = clip30(lg10(sqrt(lo)) - lg10(sqrt(up)));
      f[21] = clip30(n > 1 ? lg10(dmin) - lg10(offs / (fn * fn - fn)) : 0.0);
      f[22] = clip30(tiny / fn);
      f[23] = clip30(cgmax);
      float4* o4 = reinterpret_cast<float4*>(out + m * kFeat);
#pragma unroll
      for (int i = 0; i < kFeat / 4; ++i) o4[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
    }
    __syncwarp();
  }
}

// Inference: one thread per sample, parameters broadcast from shared memory.
__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ norm,
                                                          const float* __restrict__ X, long long batch,
                                                          float* logits, signed char* tier) {
  __shared__ float w[kParams + 2 * kFeat];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) w[i] = P[i];
  for (int i = threadIdx.x; i < 2 * kFeat; i += blockDim.x) w[kParams + i] = norm[i];
  __syncthreads();
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= batch) return;
  const float* mu = w + kParams;
  const float* isd = mu + kFeat;
  float x[kFeat];
#pragma unroll
  for (int k = 0; k < kFeat; ++k) x[k] = (X[s * kFeat + k] - mu[k]) * isd[k];
  float h1[kHid];
#pragma unroll
  for (int j = 0; j < kHid; ++j) h1[j] = w[kOffB1 + j];
#pragma unroll
  for (int k = 0; k < kFeat; ++k)
#pragma unroll
    for (int j = 0; j < kHid; ++j) h1[j] = fmaf(x[k], w[kOffW1 + k * kHid + j], h1[j]);
  float h2[kHid];
#pragma unroll
  for (int j = 0; j < kHid; ++j) {
    h1[j] = fmaxf(h1[j], 0.f);
    h2[j] = w[kOffB2 + j];
  }
#pragma unroll
  for (int k = 0; k < kHid; ++k)
#pragma unroll
    for (int j = 0; j < kHid; ++j) h2[j] = fmaf(h1[k], w[kOffW2 + k * kHid + j], h2[j]);
  float lg[kTiers];
#pragma unroll
  for (int c = 0; c < kTiers; ++c) lg[c] = w[kOffB3 + c];
#pragma unroll
  for (int k = 0; k < kHid; ++k) {
    const float h = fmaxf(h2[k], 0.f);
#pragma unroll
    for (int c = 0; c < kTiers; ++c) lg[c] = fmaf(h, w[kOffW3 + k * kTiers + c], lg[c]);
  }
  int best = 0;
#pragma unroll
  for (int c = 1; c < kTiers; ++c) best = lg[c] > lg[best] ? c : best;
  if (logits)
#pragma unroll
    for (int c = 0; c < kTiers; ++c) logits[s * kTiers + c] = lg[c];
  if (tier) tier[s] = (signed char)best;
}

// Training: a block of kTrainBlock samples runs forward and backward with its
// activations in shared memory and writes its partial gradient (kParams values)
// and partial loss to scratch; grad_reduce_kernel sums the partials in block order.
struct TrainSmem {
  float w[kParams];
  float mu[kFeat], isd[kFeat];
  float x[kTrainBlock][kFeat];
  float h1[kTrainBlock][kHid];
  float h2[kTrainBlock][kHid];
  float dh1[kTrainBlock][kHid];
  float dh2[kTrainBlock][kHid];
  float dl[kTrainBlock][kTiers];
  float loss[kTrainBlock];
};

__global__ void __launch_bounds__(kTrainThreads) mlp_train_kernel(const float* __restrict__ P,
                                                                   const float* __restrict__ norm,
                                                                   const float* __restrict__ X,
                                                                   const signed char* __restrict__ label,
                                                                   const float* __restrict__ cw, long long batch,
                                                                   float* partial) {
  extern __shared__ __align__(16) unsigned char tsm_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(tsm_raw);
  const int t = threadIdx.x;
  for (int i = t; i < kParams; i += kTrainThreads) S.w[i] = P[i];
  if (t < kFeat) {
    S.mu[t] = norm[t];
    S.isd[t] = norm[kFeat + t];
  }
  __syncthreads();
  const long long s0 = (long long)blockIdx.x * kTrainBlock;
  for (int i = t; i < kTrainBlock * kFeat; i += kTrainThreads) {
    const int s = i / kFeat, k = i % kFeat;
    S.x[s][k] = (s0 + s < batch) ? (X[(s0 + s) * kFeat + k] - S.mu[k]) * S.isd[k] : 0.f;
  }
  __syncthreads();
  const int s = t >> 2, q = t & 3;  // sample, quarter (16 hidden units each)
  const bool live = s0 + s < batch;
  // forward
#pragma unroll
  for (int jj = 0; jj < 16; ++jj) {
    const int j = q * 16 + jj;
    float a = S.w[kOffB1 + j];
#pragma unroll
    for (int k = 0; k < kFeat; ++k) a = fmaf(S.x[s][k], S.w[kOffW1 + k * kHid + j], a);
    S.h1[s][j] = live ? fmaxf(a, 0.f) : 0.f;
  }
  __syncthreads();
#pragma unroll 4
  for (int jj = 0; jj < 16; ++jj) {
    const int j = q * 16 + jj;
    float a = S.w[kOffB2 + j];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k) a = fmaf(S.h1[s][k], S.w[kOffW2 + k * kHid + j], a);
    S.h2[s][j] = live ? fmaxf(a, 0.f) : 0.f;
  }
  __syncthreads();
  {
    float a = S.w[kOffB3 + q];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k) a = fmaf(S.h2[s][k], S.w[kOffW3 + k * kTiers + q], a);
    S.dl[s][q] = a;  // logits for now
  }
  __syncthreads();
  if (q == 0) {
    float lg[kTiers], mx = -3.0e38f;
#pragma unroll
    for (int c = 0; c < kTiers; ++c) {
      lg[c] = S.dl[s][c];
      mx = fmaxf(mx, lg[c]);
    }
    float z = 0.f;
#pragma unroll
    for (int c = 0; c < kTiers; ++c) z += expf(lg[c] - mx);
    const int y = live ? (int)label[s0 + s] : 0;
    const float wy = live ? (cw ? cw[y] : 1.f) : 0.f;
    const float scale = wy / (float)batch;
#pragma unroll
    for (int c = 0; c < kTiers; ++c) {
      const float pc = expf(lg[c] - mx) / z;
      S.dl[s][c] = scale * (pc - (c == y ? 1.f : 0.f));
    }
    S.loss[s] = live ? scale * (logf(z) + mx - lg[y]) : 0.f;
  }
  __syncthreads();
  // backward through the hidden layers
#pragma unroll 4
  for (int jj = 0; jj < 16; ++jj) {
    const int j = q * 16 + jj;
    float a = 0.f;
#pragma unroll
    for (int c = 0; c < kTiers; ++c) a = fmaf(S.w[kOffW3 + j * kTiers + c], S.dl[s][c], a);
    S.dh2[s][j] = S.h2[s][j] > 0.f ? a : 0.f;
  }
  __syncthreads();
#pragma unroll 4
  for (int jj = 0; jj < 16; ++jj) {
    const int i = q * 16 + jj;
    float a = 0.f;
#pragma unroll 8
    for (int j = 0; j < kHid; ++j) a = fmaf(S.w[kOffW2 + i * kHid + j], S.dh2[s][j], a);
    S.dh1[s][i] = S.h1[s][i] > 0.f ? a : 0.f;
  }
  __syncthreads();
  // parameter gradients over the block's samples
  float* out = partial + (long long)blockIdx.x * (kParams + 1);
  for (int p = t; p < kParams; p += kTrainThreads) {
    float g = 0.f;
    if (p < kOffB1) {
      const int k = p / kHid, j = p % kHid;
      for (int ss = 0; ss < kTrainBlock; ++ss) g = fmaf(S.x[ss][k], S.dh1[ss][j], g);
    } else if (p < kOffW2) {
      const int j = p - kOffB1;
      for (int ss = 0; ss < kTrainBlock; ++ss) g += S.dh1[ss][j];
    } else if (p < kOffB2) {
      const int k = (p - kOffW2) / kHid, j = (p - kOffW2) % kHid;
      for (int ss = 0; ss < kTrainBlock; ++ss) g = fmaf(S.h1[ss][k], S.dh2[ss][j], g);
    } else if (p < kOffW3) {
      const int j = p - kOffB2;
      for (int ss = 0; ss < kTrainBlock; ++ss) g += S.dh2[ss][j];
    } else if (p < kOffB3) {
      const int k = (p - kOffW3) / kTiers, c = (p - kOffW3) % kTiers;
      for (int ss = 0; ss < kTrainBlock; ++ss) g = fmaf(S.h2[ss][k], S.dl[ss][c], g);
    } else {
      const int c = p - kOffB3;
      for (int ss = 0; ss < kTrainBlock; ++ss) g += S.dl[ss][c];
    }
    out[p] = g;
  }
  if (t == 0) {
    float l = 0.f;
    for (int ss = 0; ss < kTrainBlock; ++ss) l += S.loss[ss];
    out[kParams] = l;
  }
}

// grad[p] = sum over blocks of partial[b][p] (p = kParams is the loss), in block order.
__global__ void grad_reduce_kernel(const float* __restrict__ partial, int blocks, float* grad, float* loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kParams) return;
  float g = 0.f;
  for (int b = 0; b < blocks; ++b) g += partial[(long long)b * (kParams + 1) + p];
  if (p < kParams) grad[p] = g;
  else if (loss) *loss = g;
}

// Adam (Kingma & Ba 2015) with bias correction.
__global__ void adam_kernel(float* P, const float* __restrict__ g, float* m, float* v, long long count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace dev
}  // namespace tsdx
