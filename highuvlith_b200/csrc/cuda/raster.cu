// Pixel-aligned rectangle rasteriser: the raster of a binary Manhattan clip
// (Mask::rasterize for pixel-aligned Rect features, mask.rs:1717-1741, where
// every pixel's coverage is 0 or 1).  Dark field: clear (1) rectangles on an
// opaque (0) background; bright field: opaque rectangles on a clear field.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../../include/huv_b200.h"

namespace huv_dev {

// grid: (n / rows_per_block, clips).  Each block paints its band of rows.
__global__ void rasterize_rects(int n, int rows_per_block, const int32_t* __restrict__ rects,
                                const int32_t* __restrict__ offsets, uint8_t bg, uint8_t fg,
                                uint8_t* __restrict__ out) {
  const int clip = blockIdx.y;
  const int y0 = blockIdx.x * rows_per_block;
  const int y1 = min(n, y0 + rows_per_block);
  uint8_t* oc = out + static_cast<size_t>(clip) * n * n;
  for (int t = threadIdx.x; t < (y1 - y0) * n; t += blockDim.x)
    oc[static_cast<size_t>(y0) * n + t] = bg;
  __syncthreads();
  const int r0 = offsets[clip], r1 = offsets[clip + 1];
  for (int r = r0; r < r1; ++r) {
    const int rx = rects[4 * r], ry = rects[4 * r + 1], rw = rects[4 * r + 2], rh = rects[4 * r + 3];
    const int a = max(ry, y0), b = min(ry + rh, y1);
    const int xa = max(rx, 0), xb = min(rx + rw, n);
    if (a >= b || xa >= xb) continue;
    const int w = xb - xa;
    for (int t = threadIdx.x; t < (b - a) * w; t += blockDim.x) {
      const int yy = a + t / w, xx = xa + t % w;
      oc[static_cast<size_t>(yy) * n + xx] = fg;
    }
  }
}

}  // namespace huv_dev

extern "C" huv_status huv_rasterize_rects(int32_t n, int32_t n_clips, const int32_t* rects_dev,
                                          const int32_t* clip_offsets_dev, int32_t dark_field,
                                          uint8_t* raster_out_dev, void* stream) {
  if (n <= 0 || n_clips < 0 || (n_clips > 0 && (!rects_dev || !clip_offsets_dev || !raster_out_dev)))
    return HUV_ERR_INVALID_PARAMETER;
  if (n_clips == 0) return HUV_OK;
  const int rpb = n >= 16 ? 16 : n;
  dim3 grid((n + rpb - 1) / rpb, n_clips);
  const uint8_t bg = dark_field ? 0 : 1, fg = dark_field ? 1 : 0;
  huv_dev::rasterize_rects<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, rpb, rects_dev, clip_offsets_dev, bg, fg, raster_out_dev);
  return cudaGetLastError() == cudaSuccess ? HUV_OK : HUV_ERR_CUDA;
}
