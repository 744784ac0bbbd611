// Uneven-stream solves, float64 instantiation.
#include "stream_launch.cuh"

namespace tsdx {
namespace host {
template int run_stream<double>(dev::StreamArgs<double>, void*, long long, cudaStream_t);
}  // namespace host
}  // namespace tsdx
