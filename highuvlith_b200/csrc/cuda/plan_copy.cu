// Gather and scatter of an uneven plan's clips between the callers' own
// device buffers and a group's contiguous staging buffers, as one kernel
// per direction: clip c copies `bytes` from src[c] to dst[c] in 16-byte
// words (both pointer arrays on the device, built once per plan).  One
// launch replaces a device-to-device copy per clip, whose fixed cost
// dominates for small clips.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace huv_dev {

__global__ void plan_copy_kernel(const uint4* const* __restrict__ src, uint4* const* __restrict__ dst, size_t n16) {
  const uint4* s = src[blockIdx.y];
  uint4* d = dst[blockIdx.y];
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n16;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    d[i] = s[i];
}

}  // namespace huv_dev

namespace huv_launch {

// Copies clips [0, count) of a plan group; every pointer and `bytes` must
// be multiples of 16 (the caller checks).
cudaError_t plan_copy(const void* const* src, void* const* dst, size_t bytes, int count, cudaStream_t st) {
  if (count <= 0 || bytes == 0) return cudaSuccess;
  if (bytes % 16 != 0 || count > 65535) return cudaErrorInvalidValue;
  const size_t n16 = bytes / 16;
  const unsigned bx = static_cast<unsigned>(std::min<size_t>((n16 + 255) / 256, 64));
  huv_dev::plan_copy_kernel<<<dim3(bx, static_cast<unsigned>(count)), 256, 0, st>>>(
      reinterpret_cast<const uint4* const*>(src), reinterpret_cast<uint4* const*>(dst), n16);
  return cudaGetLastError();
}

}  // namespace huv_launch
