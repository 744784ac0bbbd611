// Uneven-stream solves, float32 instantiation.
#include "stream_launch.cuh"

namespace tsdx {
namespace host {
long long stream_scratch_bytes(long long count) { return stream_scratch_bytes_of(count); }
template int run_stream<float>(dev::StreamArgs<float>, void*, long long, cudaStream_t);
}  // namespace host
}  // namespace tsdx
