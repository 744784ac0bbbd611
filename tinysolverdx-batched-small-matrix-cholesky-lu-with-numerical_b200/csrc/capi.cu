// C-ABI of the batched solver (declared in include/tsdx_cuda.h).
//
// Device-pointer entry points validate their arguments exactly like the
// reference's batch drivers (batched.hpp:39-43, :184) and enqueue one fused
// kernel per pass of at most 8 right-hand sides. Host-pointer entry points
// replace the reference's synchronous CUDA backend (cuda_backend.cu:155-188):
// they stream the batch through a cached device workspace in chunks, with the
// host->device copy of one chunk, the kernel of the previous one and the
// device->host copy of the one before that in flight at the same time.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tsdx_cuda.h"
#include "launch.cuh"
#include "stream.cuh"

namespace tsdx {
namespace host {

int run_ir(bool spd, const double* A, int n, long long batch, double* B, const signed char* tier, int default_tier,
           int itmax, double tol, int* info, int* status, double* bwd, cudaStream_t st);
long long stream_scratch_bytes(long long count);
template <class T> int run_stream(dev::StreamArgs<T> a, void* scratch, long long scratch_bytes, cudaStream_t st);

namespace {
thread_local std::string g_err;
std::atomic<long long> g_launches{0};
int g_sms[kMaxDevices] = {0};
}  // namespace

void set_cuda_error(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
}
void set_error_message(const std::string& msg) { g_err = msg; }
std::atomic<long long>& launch_counter() { return g_launches; }

int lu_kernel_family() {
  static const int fam = [] {
    const char* e = std::getenv("TSDX_LU_KERNEL");
    const std::string v = e ? e : "";
    return v == "tc" ? 3 : v == "smem" ? 1 : 0;
  }();
  return fam;
}

int device_sms(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return 148;
  if (g_sms[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    g_sms[dev] = v;
  }
  return g_sms[dev];
}

namespace {

enum Kind { POTRF, GETRF, POTRS, GETRS, POSV, GESV };

inline int check_common(int n, int64_t batch, int nrhs) {
  if (n < 1 || n > 64) return TSDX_ERR_N;
  if (batch < 0) return TSDX_ERR_BATCH;
  if (nrhs < 0) return TSDX_ERR_NRHS;
  return TSDX_OK;
}
template <class T> inline bool aligned(const T* p) { return reinterpret_cast<uintptr_t>(p) % alignof(T) == 0; }

// ---- device-pointer implementation --------------------------------------------
template <class T>
int run_device(Kind kind, T* A, const int* piv_in, int n, int64_t batch, T* B, int nrhs, int* piv, int* info,
               cudaStream_t st) {
  if (int rc = check_common(n, batch, nrhs)) return rc;
  const bool has_b = (kind == POTRS || kind == GETRS || kind == POSV || kind == GESV);
  if (!has_b) nrhs = 0;
  if (!A || !aligned(A)) return TSDX_ERR_NULL;
  if ((kind == GETRF || kind == GESV) && !piv) return TSDX_ERR_NULL;
  if (kind == GETRS && !piv_in) return TSDX_ERR_NULL;
  if (has_b && nrhs > 0 && (!B || !aligned(B))) return TSDX_ERR_NULL;
  if (batch == 0) return TSDX_OK;

  dev::SolveArgs<T> a{};
  a.A = A;
  a.B = B;
  a.piv = (kind == GETRS) ? const_cast<int*>(piv_in) : piv;
  a.info = info;
  a.batch = batch;
  a.n = n;
  a.ldb = nrhs;
  a.status = nullptr;
  a.wf = 1;
  if (kind == POTRF || kind == GETRF || kind == POSV || kind == GESV) {
    a.b0 = 0;
    a.nrhs = std::min(nrhs, 8);
    const int rc = (kind == POTRF || kind == POSV) ? run_chol<T>(a, st) : run_lu<T>(a, st);
    if (rc) return rc;
    for (int b0 = 8; b0 < nrhs; b0 += 8) {  // remaining right-hand sides from the factor
      a.b0 = b0;
      a.nrhs = std::min(8, nrhs - b0);
      const int r2 = (kind == POSV) ? run_potrs<T>(a, st) : run_getrs<T>(a, st);
      if (r2) return r2;
    }
    return TSDX_OK;
  }
  for (int b0 = 0; b0 < nrhs; b0 += 8) {
    a.b0 = b0;
    a.nrhs = std::min(8, nrhs - b0);
    const int rc = (kind == POTRS) ? run_potrs<T>(a, st) : run_getrs<T>(a, st);
    if (rc) return rc;
  }
  return TSDX_OK;
}

// ---- host-pointer implementation ----------------------------------------------
constexpr int kSlots = 3;
constexpr size_t kChunkBytes = size_t(96) << 20;  // A bytes per chunk, at most
// A small batch is still cut into kMinChunks chunks (of at least kMinChunkBytes), so
// that its copies overlap too: with two chunks, most of the transfer would run alone.
constexpr int kMinChunks = 8;
constexpr size_t kMinChunkBytes = size_t(4) << 20;

struct Slot {
  void* a = nullptr;
  void* b = nullptr;
  int* piv = nullptr;
  int* info = nullptr;
  size_t acap = 0, bcap = 0, pcap = 0, icap = 0;
  cudaStream_t st = nullptr;
};
struct DeviceCtx {
  Slot slot[kSlots];
  bool init = false;
};
std::mutex g_host_mu;
DeviceCtx g_ctx[tsdx::host::kMaxDevices];

int grow(void** p, size_t* cap, size_t need) {
  if (need <= *cap) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, need);
  if (e != cudaSuccess) { set_cuda_error(e, "cudaMalloc"); return TSDX_ERR_CUDA; }
  *cap = need;
  return 0;
}

#define TSDX_CK(call, what)                                          \
  do {                                                               \
    cudaError_t e_ = (call);                                         \
    if (e_ != cudaSuccess) { set_cuda_error(e_, what); return TSDX_ERR_CUDA; } \
  } while (0)

// keep_a: the one-shot solve leaves the caller's A untouched and returns no pivots
// (the reference's Python-level gesv/posv return only (x, info), __init__.py:102-111).
template <class T>
int run_host(Kind kind, T* A, const int* piv_in, int n, int64_t batch, T* B, int nrhs, int* piv, int* info,
             bool keep_a = false) {
  if (int rc = check_common(n, batch, nrhs)) return rc;
  const bool has_b = (kind == POTRS || kind == GETRS || kind == POSV || kind == GESV);
  if (!has_b) nrhs = 0;
  if (!A) return TSDX_ERR_NULL;
  if ((kind == GETRF || kind == GESV) && !piv && !keep_a) return TSDX_ERR_NULL;
  if (kind == GETRS && !piv_in) return TSDX_ERR_NULL;
  if (has_b && nrhs > 0 && !B) return TSDX_ERR_NULL;
  if (batch == 0) return TSDX_OK;
  int devi = 0;
  if (cudaGetDevice(&devi) != cudaSuccess) return TSDX_ERR_NODEV;
  if (devi >= tsdx::host::kMaxDevices) return TSDX_ERR_NODEV;

  std::lock_guard<std::mutex> lock(g_host_mu);
  DeviceCtx& ctx = g_ctx[devi];
  if (!ctx.init) {
    for (auto& s : ctx.slot) TSDX_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx.init = true;
  }
  const size_t mat = size_t(n) * n * sizeof(T), rhs = size_t(n) * nrhs * sizeof(T);
  const size_t target = std::min(kChunkBytes, std::max(kMinChunkBytes, mat * size_t(batch) / kMinChunks));
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(batch, int64_t(target / mat)));
  for (auto& s : ctx.slot) {
    if (int rc = grow(&s.a, &s.acap, mat * chunk)) return rc;
    if (has_b && nrhs > 0)
      if (int rc = grow(&s.b, &s.bcap, rhs * chunk)) return rc;
    if (kind == GETRF || kind == GESV || kind == GETRS)
      if (int rc = grow(reinterpret_cast<void**>(&s.piv), &s.pcap, size_t(n) * chunk * sizeof(int))) return rc;
    if (info)
      if (int rc = grow(reinterpret_cast<void**>(&s.info), &s.icap, size_t(chunk) * sizeof(int))) return rc;
  }
  const bool writes_a = (kind == POTRF || kind == GETRF || kind == POSV || kind == GESV) && !keep_a;
  const bool writes_piv = (kind == GETRF || kind == GESV) && !keep_a;
  const bool writes_info = info && (kind == POTRF || kind == GETRF || kind == POSV || kind == GESV);
  auto enqueue = [&]() -> int {
    int c = 0;
    for (int64_t m = 0; m < batch; m += chunk, ++c) {
      Slot& s = ctx.slot[c % kSlots];
      const int64_t cnt = std::min(chunk, batch - m);
      T* dA = static_cast<T*>(s.a);
      T* dB = static_cast<T*>(s.b);
      TSDX_CK(cudaMemcpyAsync(dA, reinterpret_cast<const char*>(A) + m * mat, mat * cnt, cudaMemcpyHostToDevice, s.st), "H2D A");
      if (has_b && nrhs > 0)
        TSDX_CK(cudaMemcpyAsync(dB, reinterpret_cast<const char*>(B) + m * rhs, rhs * cnt, cudaMemcpyHostToDevice, s.st), "H2D B");
      if (kind == GETRS)
        TSDX_CK(cudaMemcpyAsync(s.piv, piv_in + m * n, size_t(n) * cnt * sizeof(int), cudaMemcpyHostToDevice, s.st), "H2D piv");
      // the device workspace copy of A may take the factor even when the caller's A is kept
      const int rc = run_device<T>(kind, dA, s.piv, n, cnt, dB, nrhs, s.piv, writes_info ? s.info : nullptr, s.st);
      if (rc) return rc;
      if (writes_a)
        TSDX_CK(cudaMemcpyAsync(reinterpret_cast<char*>(A) + m * mat, dA, mat * cnt, cudaMemcpyDeviceToHost, s.st), "D2H A");
      if (has_b && nrhs > 0)
        TSDX_CK(cudaMemcpyAsync(reinterpret_cast<char*>(B) + m * rhs, dB, rhs * cnt, cudaMemcpyDeviceToHost, s.st), "D2H B");
      if (writes_piv)
        TSDX_CK(cudaMemcpyAsync(piv + m * n, s.piv, size_t(n) * cnt * sizeof(int), cudaMemcpyDeviceToHost, s.st), "D2H piv");
      if (writes_info)
        TSDX_CK(cudaMemcpyAsync(info + m, s.info, size_t(cnt) * sizeof(int), cudaMemcpyDeviceToHost, s.st), "D2H info");
    }
    return TSDX_OK;
  };
  // drain the slots' streams on failure too: no copy into the caller's buffers outlives the call
  int rc = enqueue();
  for (auto& s : ctx.slot) {
    const cudaError_t e = cudaStreamSynchronize(s.st);
    if (e != cudaSuccess && rc == TSDX_OK) {
      set_cuda_error(e, "cudaStreamSynchronize");
      rc = TSDX_ERR_CUDA;
    }
  }
  return rc;
}

}  // namespace
}  // namespace host
}  // namespace tsdx

using tsdx::host::GESV;
using tsdx::host::GETRF;
using tsdx::host::GETRS;
using tsdx::host::POSV;
using tsdx::host::POTRF;
using tsdx::host::POTRS;
using tsdx::host::run_device;
using tsdx::host::run_host;

#define API extern "C" __attribute__((visibility("default")))
#define ST(s) static_cast<cudaStream_t>(s)

API int tsdx_cuda_available(void) {
  int c = 0;
  return cudaGetDeviceCount(&c) == cudaSuccess && c > 0 ? 1 : 0;
}
API const char* tsdx_cuda_last_error(void) { return tsdx::host::g_err.c_str(); }
API int64_t tsdx_cuda_launch_count(void) { return tsdx::host::launch_counter().load(); }

// Self-check of the Markstein-corrected division used by the kernels (common.cuh
// div_by) against the IEEE division, element by element. Not part of the solver
// API; the test-suite calls it on adversarial operand sets.
namespace {
template <class T>
__global__ void div_check_kernel(const T* a, const T* b, T* fast, T* ieee, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const T y = tsdx::dev::rcp_(b[i]);
  fast[i] = tsdx::dev::div_by(a[i], b[i], y);
  ieee[i] = tsdx::dev::div_(a[i], b[i]);
}
template <class T>
int div_check(const T* a, const T* b, T* fast, T* ieee, int64_t count, void* st) {
  if (count <= 0) return TSDX_OK;
  div_check_kernel<T><<<(unsigned)((count + 255) / 256), 256, 0, ST(st)>>>(a, b, fast, ieee, count);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { tsdx::host::set_cuda_error(e, "kernel launch"); return TSDX_ERR_CUDA; }
  return TSDX_OK;
}
}  // namespace
API int tsdx_internal_div_check_f64(const double* a, const double* b, double* fast, double* ieee, int64_t count,
                                     void* st) {
  return div_check<double>(a, b, fast, ieee, count, st);
}
API int tsdx_internal_div_check_f32(const float* a, const float* b, float* fast, float* ieee, int64_t count,
                                     void* st) {
  return div_check<float>(a, b, fast, ieee, count, st);
}

// ---- mixed precision + iterative refinement ------------------------------------
namespace {
int ir_entry(bool spd, const double* A, int n, int64_t batch, double* B, const signed char* tier, int default_tier,
             int itmax, double tol, int* info, int* status, double* bwd, void* st) {
  if (n < 1 || n > 64) return TSDX_ERR_N;
  if (batch < 0) return TSDX_ERR_BATCH;
  if (!A || !B) return TSDX_ERR_NULL;
  if (default_tier < 0 || default_tier > 3 || itmax < 0 || !(tol > 0.0)) return TSDX_ERR_NRHS;
  if (batch == 0) return TSDX_OK;
  cudaStream_t s = ST(st);
  int* stat = status;
  if (!stat) {
    // the fallback pass needs the per-matrix status; stream-ordered scratch when the caller has none
    const cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&stat), size_t(batch) * sizeof(int), s);
    if (e != cudaSuccess) { tsdx::host::set_cuda_error(e, "cudaMallocAsync"); return TSDX_ERR_CUDA; }
  }
  int rc = tsdx::host::run_ir(spd, A, n, batch, B, tier, default_tier, itmax, tol, info, stat, bwd, s);
  if (!status) {
    const cudaError_t e = cudaFreeAsync(stat, s);
    if (e != cudaSuccess && rc == 0) { tsdx::host::set_cuda_error(e, "cudaFreeAsync"); rc = TSDX_ERR_CUDA; }
  }
  return rc;
}
}  // namespace

API int tsdx_cuda_gesv_ir_f64(const double* A, int n, int64_t batch, double* B, const signed char* tier,
                              int default_tier, int itmax, double tol, int* info, int* status, double* bwd,
                              void* stream) {
  return ir_entry(false, A, n, batch, B, tier, default_tier, itmax, tol, info, status, bwd, stream);
}
API int tsdx_cuda_posv_ir_f64(const double* A, int n, int64_t batch, double* B, const signed char* tier,
                              int default_tier, int itmax, double tol, int* info, int* status, double* bwd,
                              void* stream) {
  return ir_entry(true, A, n, batch, B, tier, default_tier, itmax, tol, info, status, bwd, stream);
}

// ---- uneven stream -------------------------------------------------------------
API int64_t tsdx_cuda_stream_scratch_bytes(int64_t count) {
  return count < 0 ? 0 : tsdx::host::stream_scratch_bytes(count);
}
namespace {
template <class T>
int stream_entry(T* A, const int64_t* aoff, T* B, const int64_t* boff, int* piv, const int64_t* poff, int* info,
                 const int* n, const int* nrhs, const signed char* kind, int64_t count, int write_factors,
                 unsigned sched, void* scratch, int64_t scratch_bytes, void* st) {
  if (count < 0 || count > (int64_t(1) << 31) - 1) return TSDX_ERR_BATCH;
  if (count == 0) return TSDX_OK;
  if (!A || !aoff || !n || !nrhs || !kind) return TSDX_ERR_NULL;
  if (write_factors && (!piv || !poff)) return TSDX_ERR_NULL;
  tsdx::dev::StreamArgs<T> a{};
  a.A = A;
  a.B = B;
  a.piv = piv;
  a.info = info;
  a.aoff = reinterpret_cast<const long long*>(aoff);
  a.boff = reinterpret_cast<const long long*>(boff);
  a.poff = reinterpret_cast<const long long*>(poff);
  a.n = n;
  a.nrhs = nrhs;
  a.kind = kind;
  a.count = (int)count;
  a.wf = write_factors ? 1 : 0;
  a.sched = sched;
  if (B && !boff) return TSDX_ERR_NULL;
  return tsdx::host::run_stream<T>(a, scratch, scratch_bytes, ST(st));
}

// ---- uneven stream from host memory ------------------------------------------------
// The packed set is cut into chunks of about kStreamChunkBytes, in index order, counting
// every byte a matrix moves or occupies (A, B, pivots, info, its metadata record and
// sort scratch). A chunk travels with its own metadata record (offsets rebased to the
// chunk's first matrix, orders, right-hand-side counts, kinds), so the device holds
// kStreamSlots chunks at a time whatever the size of the set, and chunk c's host->device
// copy, chunk c-1's sort and drain and chunk c-2's device->host copy run at the same time
// on the slots' streams. One host pass validates every entry and cuts the chunks before
// anything is copied. Each slot has one pinned record buffer: chunk c's record is
// written into it once chunk c - kStreamSlots's record upload has finished (an event),
// just before chunk c's copies are queued, so pinned memory is bounded by the chunk
// size too.
constexpr int kStreamSlots = 3;
constexpr size_t kStreamChunkBytes = size_t(96) << 20;

struct StreamSlotWs {
  void* a = nullptr;
  void* b = nullptr;
  int* piv = nullptr;
  int* info = nullptr;
  void* meta = nullptr;  // metadata record, then the sort scratch
  size_t acap = 0, bcap = 0, pcap = 0, icap = 0, mcap = 0;
  cudaStream_t st = nullptr;
};
struct StreamHostCtx {
  StreamSlotWs ws[kStreamSlots];
  bool init = false;
  void* hrec[kStreamSlots] = {};            // pinned record buffer of each slot
  cudaEvent_t rec_sent[kStreamSlots] = {};  // the slot's last record upload has finished
  size_t hcap = 0;
};
StreamHostCtx g_stream_ctx[tsdx::host::kMaxDevices];

// record of cnt matrices: aoff, boff, poff (int64), n, nrhs (int32), kind (int8)
constexpr size_t meta_record_bytes(int64_t cnt) { return (size_t(cnt) * 33 + 255) / 256 * 256; }
// host and device bytes of one matrix beyond its A, B and pivots: record, info, sort scratch
constexpr size_t kStreamPerMatrixBytes = 33 + 4 + 4;

template <class T>
int stream_host_entry(T* A, T* B, int* piv, int* info, const int* n, const int* nrhs, const signed char* kind,
                      int64_t count, int write_factors, unsigned sched) {
  using tsdx::host::set_cuda_error;
  if (count < 0 || count > (int64_t(1) << 31) - 1) return TSDX_ERR_BATCH;
  if (count == 0) return TSDX_OK;
  if (!A || !n || !nrhs || !kind) return TSDX_ERR_NULL;
  if (write_factors && !piv) return TSDX_ERR_NULL;

  // chunk c: matrices first[c] .. first[c+1]-1 holding ext[c] = {A, B, pivot} elements
  struct Ext {
    int64_t a, b, p;
  };
  std::vector<int64_t> first;
  std::vector<Ext> ext;
  int64_t mx_cnt = 0, mx_a = 0, mx_b = 0, mx_p = 0;
  bool any_b = false;
  {
    int64_t i0 = 0, a = 0, b = 0, p = 0;
    size_t bytes = 0;
    for (int64_t i = 0; i < count; ++i) {
      const int ni = n[i], ri = nrhs[i];
      if (ni < 1 || ni > 64) return TSDX_ERR_N;
      if (ri < 0 || ri > 8) return TSDX_ERR_NRHS;
      a += int64_t(ni) * ni;
      b += int64_t(ni) * ri;
      p += ni;
      bytes += size_t(ni) * (ni + ri) * sizeof(T) + size_t(ni) * sizeof(int) + kStreamPerMatrixBytes;
      if (bytes >= kStreamChunkBytes || i + 1 == count) {
        first.push_back(i0);
        ext.push_back({a, b, p});
        mx_cnt = std::max(mx_cnt, i + 1 - i0);
        mx_a = std::max(mx_a, a);
        mx_b = std::max(mx_b, b);
        mx_p = std::max(mx_p, p);
        any_b = any_b || b > 0;
        i0 = i + 1;
        a = b = p = 0;
        bytes = 0;
      }
    }
    first.push_back(count);
  }
  if (any_b && !B) return TSDX_ERR_NULL;
  int devi = 0;
  if (cudaGetDevice(&devi) != cudaSuccess) return TSDX_ERR_NODEV;
  if (devi >= tsdx::host::kMaxDevices) return TSDX_ERR_NODEV;

  std::lock_guard<std::mutex> lock(tsdx::host::g_host_mu);
  StreamHostCtx& sc = g_stream_ctx[devi];
  if (!sc.init) {
    for (auto& w : sc.ws) TSDX_CK(cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : sc.rec_sent) TSDX_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    sc.init = true;
  }
  const size_t scratch_bytes = size_t(tsdx::host::stream_scratch_bytes(mx_cnt));
  for (auto& w : sc.ws) {
    using tsdx::host::grow;
    if (int rc = grow(&w.a, &w.acap, size_t(mx_a) * sizeof(T))) return rc;
    if (any_b)
      if (int rc = grow(&w.b, &w.bcap, size_t(mx_b) * sizeof(T))) return rc;
    if (write_factors)
      if (int rc = grow(reinterpret_cast<void**>(&w.piv), &w.pcap, size_t(mx_p) * sizeof(int))) return rc;
    if (info)
      if (int rc = grow(reinterpret_cast<void**>(&w.info), &w.icap, size_t(mx_cnt) * sizeof(int))) return rc;
    if (int rc = grow(&w.meta, &w.mcap, meta_record_bytes(mx_cnt) + scratch_bytes)) return rc;
  }
  if (meta_record_bytes(mx_cnt) > sc.hcap) {
    // the previous call synchronized its streams before returning: nothing reads the old buffers
    for (auto& h : sc.hrec) {
      if (h) cudaFreeHost(h);
      h = nullptr;
    }
    sc.hcap = 0;
    for (auto& h : sc.hrec) TSDX_CK(cudaMallocHost(&h, meta_record_bytes(mx_cnt)), "cudaMallocHost");
    sc.hcap = meta_record_bytes(mx_cnt);
  }

  const int nchunks = int(first.size()) - 1;
  auto enqueue = [&]() -> int {
    int64_t a0 = 0, b0 = 0, p0 = 0;
    for (int c = 0; c < nchunks; ++c) {
      const int64_t i0 = first[c], cnt = first[c + 1] - i0;
      const int64_t ca = ext[c].a, cb = ext[c].b, cp = ext[c].p;
      const int k = c % kStreamSlots;
      unsigned char* rec = static_cast<unsigned char*>(sc.hrec[k]);
      // this chunk's record, once the slot's previous record has reached the device
      if (c >= kStreamSlots) TSDX_CK(cudaEventSynchronize(sc.rec_sent[k]), "cudaEventSynchronize");
      {
        int64_t* ao = reinterpret_cast<int64_t*>(rec);
        int64_t* bo = ao + cnt;
        int64_t* po = bo + cnt;
        int* nn = reinterpret_cast<int*>(po + cnt);
        int* rr = nn + cnt;
        signed char* kk = reinterpret_cast<signed char*>(rr + cnt);
        int64_t a = 0, b = 0, p = 0;
        for (int64_t j = 0; j < cnt; ++j) {
          const int ni = n[i0 + j], ri = nrhs[i0 + j];
          ao[j] = a;
          bo[j] = b;
          po[j] = p;
          nn[j] = ni;
          rr[j] = ri;
          kk[j] = kind[i0 + j];
          a += int64_t(ni) * ni;
          b += int64_t(ni) * ri;
          p += ni;
        }
      }
      const StreamSlotWs& w = sc.ws[k];
      const cudaStream_t st = w.st;
      const size_t rb = meta_record_bytes(cnt);
      unsigned char* dm = static_cast<unsigned char*>(w.meta);
      TSDX_CK(cudaMemcpyAsync(dm, rec, size_t(cnt) * 33, cudaMemcpyHostToDevice, st), "H2D stream record");
      TSDX_CK(cudaEventRecord(sc.rec_sent[k], st), "cudaEventRecord");
      TSDX_CK(cudaMemcpyAsync(w.a, A + a0, size_t(ca) * sizeof(T), cudaMemcpyHostToDevice, st), "H2D A");
      if (cb > 0) TSDX_CK(cudaMemcpyAsync(w.b, B + b0, size_t(cb) * sizeof(T), cudaMemcpyHostToDevice, st), "H2D B");
      // the solve writes no pivots for Cholesky matrices: their slots go in and come
      // back unchanged, as the device call leaves them
      if (write_factors)
        TSDX_CK(cudaMemcpyAsync(w.piv, piv + p0, size_t(cp) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D piv");
      tsdx::dev::StreamArgs<T> s{};
      s.A = static_cast<T*>(w.a);
      s.B = cb > 0 ? static_cast<T*>(w.b) : nullptr;
      s.piv = write_factors ? w.piv : nullptr;
      s.info = info ? w.info : nullptr;
      s.aoff = reinterpret_cast<const long long*>(dm);
      s.boff = s.aoff + cnt;
      s.poff = s.boff + cnt;
      s.n = reinterpret_cast<const int*>(s.poff + cnt);
      s.nrhs = s.n + cnt;
      s.kind = reinterpret_cast<const signed char*>(s.nrhs + cnt);
      s.count = int(cnt);
      s.wf = write_factors ? 1 : 0;
      s.sched = sched;
      if (int rc = tsdx::host::run_stream<T>(s, dm + rb, (long long)scratch_bytes, st)) return rc;
      if (write_factors) {
        TSDX_CK(cudaMemcpyAsync(A + a0, w.a, size_t(ca) * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H A");
        TSDX_CK(cudaMemcpyAsync(piv + p0, w.piv, size_t(cp) * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H piv");
      }
      if (cb > 0) TSDX_CK(cudaMemcpyAsync(B + b0, w.b, size_t(cb) * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H B");
      if (info)
        TSDX_CK(cudaMemcpyAsync(info + i0, w.info, size_t(cnt) * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H info");
      a0 += ca;
      b0 += cb;
      p0 += cp;
    }
    return TSDX_OK;
  };
  // drain the slots' streams on failure too: no copy into the caller's buffers outlives the call
  int rc = enqueue();
  for (auto& w : sc.ws) {
    const cudaError_t e = cudaStreamSynchronize(w.st);
    if (e != cudaSuccess && rc == TSDX_OK) {
      set_cuda_error(e, "cudaStreamSynchronize");
      rc = TSDX_ERR_CUDA;
    }
  }
  return rc;
}
}  // namespace
API int tsdx_cuda_solve_stream_f32(float* A, const int64_t* aoff, float* B, const int64_t* boff, int* piv,
                                   const int64_t* poff, int* info, const int* n, const int* nrhs,
                                   const signed char* kind, int64_t count, int write_factors, unsigned sched,
                                   void* scratch, int64_t scratch_bytes, void* stream) {
  return stream_entry<float>(A, aoff, B, boff, piv, poff, info, n, nrhs, kind, count, write_factors, sched, scratch,
                             scratch_bytes, stream);
}
API int tsdx_cuda_solve_stream_f64(double* A, const int64_t* aoff, double* B, const int64_t* boff, int* piv,
                                   const int64_t* poff, int* info, const int* n, const int* nrhs,
                                   const signed char* kind, int64_t count, int write_factors, unsigned sched,
                                   void* scratch, int64_t scratch_bytes, void* stream) {
  return stream_entry<double>(A, aoff, B, boff, piv, poff, info, n, nrhs, kind, count, write_factors, sched, scratch,
                              scratch_bytes, stream);
}
API int tsdx_cuda_solve_stream_host_f32(float* A, float* B, int* piv, int* info, const int* n, const int* nrhs,
                                        const signed char* kind, int64_t count, int write_factors, unsigned sched) {
  return stream_host_entry<float>(A, B, piv, info, n, nrhs, kind, count, write_factors, sched);
}
API int tsdx_cuda_solve_stream_host_f64(double* A, double* B, int* piv, int* info, const int* n, const int* nrhs,
                                        const signed char* kind, int64_t count, int write_factors, unsigned sched) {
  return stream_host_entry<double>(A, B, piv, info, n, nrhs, kind, count, write_factors, sched);
}

#define TSDX_DEFINE(T, S)                                                                                      \
  API int tsdx_cuda_potrf_##S(T* A, int n, int64_t batch, int* info, void* st) {                               \
    return run_device<T>(POTRF, A, nullptr, n, batch, nullptr, 0, nullptr, info, ST(st));                      \
  }                                                                                                            \
  API int tsdx_cuda_getrf_##S(T* A, int n, int64_t batch, int* piv, int* info, void* st) {                     \
    return run_device<T>(GETRF, A, nullptr, n, batch, nullptr, 0, piv, info, ST(st));                          \
  }                                                                                                            \
  API int tsdx_cuda_potrs_##S(const T* L, int n, int64_t batch, T* B, int nrhs, void* st) {                    \
    return run_device<T>(POTRS, const_cast<T*>(L), nullptr, n, batch, B, nrhs, nullptr, nullptr, ST(st));      \
  }                                                                                                            \
  API int tsdx_cuda_getrs_##S(const T* LU, const int* piv, int n, int64_t batch, T* B, int nrhs, void* st) {   \
    return run_device<T>(GETRS, const_cast<T*>(LU), piv, n, batch, B, nrhs, nullptr, nullptr, ST(st));         \
  }                                                                                                            \
  API int tsdx_cuda_posv_##S(T* A, int n, int64_t batch, T* B, int nrhs, int* info, void* st) {                \
    return run_device<T>(POSV, A, nullptr, n, batch, B, nrhs, nullptr, info, ST(st));                          \
  }                                                                                                            \
  API int tsdx_cuda_gesv_##S(T* A, int n, int64_t batch, T* B, int nrhs, int* piv, int* info, void* st) {      \
    return run_device<T>(GESV, A, nullptr, n, batch, B, nrhs, piv, info, ST(st));                              \
  }                                                                                                            \
  API int tsdx_cuda_cholesky_batched_host_##S(T* A, int n, int64_t batch, int* info) {                         \
    return run_host<T>(POTRF, A, nullptr, n, batch, nullptr, 0, nullptr, info);                                \
  }                                                                                                            \
  API int tsdx_cuda_lu_batched_host_##S(T* A, int n, int64_t batch, int* piv, int* info) {                     \
    return run_host<T>(GETRF, A, nullptr, n, batch, nullptr, 0, piv, info);                                    \
  }                                                                                                            \
  API int tsdx_cuda_cholesky_solve_batched_host_##S(const T* L, int n, int64_t batch, T* B, int nrhs) {        \
    return run_host<T>(POTRS, const_cast<T*>(L), nullptr, n, batch, B, nrhs, nullptr, nullptr);                \
  }                                                                                                            \
  API int tsdx_cuda_lu_solve_batched_host_##S(const T* LU, const int* piv, int n, int64_t batch, T* B,         \
                                               int nrhs) {                                                     \
    return run_host<T>(GETRS, const_cast<T*>(LU), piv, n, batch, B, nrhs, nullptr, nullptr);                   \
  }                                                                                                            \
  API int tsdx_cuda_posv_batched_host_##S(T* A, int n, int64_t batch, T* B, int nrhs, int* info) {             \
    return run_host<T>(POSV, A, nullptr, n, batch, B, nrhs, nullptr, info);                                    \
  }                                                                                                            \
  API int tsdx_cuda_gesv_batched_host_##S(T* A, int n, int64_t batch, T* B, int nrhs, int* piv, int* info) {   \
    return run_host<T>(GESV, A, nullptr, n, batch, B, nrhs, piv, info);                                        \
  }                                                                                                            \
  API int tsdx_cuda_gesv_solve_host_##S(const T* A, int n, int64_t batch, T* B, int nrhs, int* info) {         \
    return run_host<T>(GESV, const_cast<T*>(A), nullptr, n, batch, B, nrhs, nullptr, info, true);              \
  }                                                                                                            \
  API int tsdx_cuda_posv_solve_host_##S(const T* A, int n, int64_t batch, T* B, int nrhs, int* info) {         \
    return run_host<T>(POSV, const_cast<T*>(A), nullptr, n, batch, B, nrhs, nullptr, info, true);              \
  }

TSDX_DEFINE(float, f32)
TSDX_DEFINE(double, f64)
