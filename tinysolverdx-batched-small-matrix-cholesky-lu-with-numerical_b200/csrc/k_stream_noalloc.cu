// tsdx_cuda_solve_stream_noalloc_f32: the float32 uneven-stream solve with its
// scratch in a fixed device array of this module instead of caller memory or an
// allocation on the stream. It has no TinySolverDx counterpart.
//
// Who needs it: callers that may not allocate device memory at call time. A host
// application whose memory is owned by another allocator (a framework's caching
// pool, a serving process that reserves all device memory up front) cannot hand
// out cudaMalloc'd scratch without going around that owner, and a latency-bound
// caller cannot afford cudaMalloc/cudaFree, which may synchronise the device or
// fail under memory pressure in the middle of a request. Those callers pass only
// their inputs and outputs here.
//
// Cost: every GPU that loads the library holds the array (about 1 MiB) until the
// process exits, whether or not this entry point is ever called.
//
// Scratch: kNoAllocMaxCount matrices at most (262,144; 1 MiB of sort permutation
// plus 520 bytes of bucket counters). Its device address is looked up once per
// device with cudaGetSymbolAddress on the first call on that device (that first
// call must not be made while its stream is being captured) and kept for the life
// of the process: it does not survive cudaDeviceReset, so after a reset of a device
// this entry point must not be called on it again in the same process. A larger
// count is rejected with TSDX_ERR_TOO_LARGE before anything is launched.
//
// What must start at zero: the per-bucket counters (the first kStreamBuckets ints).
// Every call zeroes them itself with cudaMemsetAsync on its stream before the
// histogram, and the scan kernel resets the queue head, so no state carries over
// from one call to the next. All other words are written before they are read.
//
// Overlapping calls race: every call on a device uses the same array, so two calls
// whose executions overlap (different streams, or different host threads) corrupt
// each other's sort. Calls must be ordered, e.g. all on one stream.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "stream_launch.cuh"

namespace tsdx {
namespace host {
void set_error_message(const std::string& msg);  // capi.cu
// compiled once, in k_stream_f32.cu
extern template int run_stream<float>(dev::StreamArgs<float>, void*, long long, cudaStream_t);
}  // namespace host
}  // namespace tsdx

namespace {

constexpr long long kNoAllocMaxCount = 1LL << 18;
constexpr long long kNoAllocBytes = tsdx::host::stream_scratch_bytes_of(kNoAllocMaxCount);

static __device__ __align__(256) int g_stream_scratch[kNoAllocBytes / sizeof(int)];

using tsdx::host::kMaxDevices;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { tsdx::host::set_cuda_error(e, "cudaGetDevice"); return TSDX_ERR_CUDA; }
  if (dev < 0 || dev >= kMaxDevices) return TSDX_ERR_NODEV;  // as every other entry point
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    e = cudaGetSymbolAddress(&g_addr[dev], g_stream_scratch);
    if (e != cudaSuccess) {
      g_addr[dev] = nullptr;
      tsdx::host::set_cuda_error(e, "cudaGetSymbolAddress");
      return TSDX_ERR_CUDA;
    }
  }
  *out = g_addr[dev];
  return TSDX_OK;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int tsdx_cuda_solve_stream_noalloc_f32(
    float* A, const int64_t* aoff, float* B, const int64_t* boff, int* piv, const int64_t* poff, int* info,
    const int* n, const int* nrhs, const signed char* kind, int64_t count, int write_factors, unsigned sched,
    void* stream) {
  if (count < 0) return TSDX_ERR_BATCH;
  if (count > kNoAllocMaxCount) {
    tsdx::host::set_error_message("count " + std::to_string(count) +
                                  " exceeds the static stream scratch capacity of " +
                                  std::to_string(kNoAllocMaxCount) + " matrices");
    return TSDX_ERR_TOO_LARGE;
  }
  if (count == 0) return TSDX_OK;
  if (!A || !aoff || !n || !nrhs || !kind) return TSDX_ERR_NULL;
  if (write_factors && (!piv || !poff)) return TSDX_ERR_NULL;
  if (B && !boff) return TSDX_ERR_NULL;
  void* scratch = nullptr;
  if (int rc = scratch_address(&scratch)) return rc;
  tsdx::dev::StreamArgs<float> a{};
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
  return tsdx::host::run_stream<float>(a, scratch, kNoAllocBytes, static_cast<cudaStream_t>(stream));
}
