// Block-cooperative Stockham FFT in shared memory (FP32 complex).
//
// S sequences of length L = 2^lg sit contiguously in a shared buffer
// (seq s at [s*L, s*L + L)).  All threads of the block take part: each pass
// maps the S*L/R butterflies of radix R over the threads, a radix-2 pass
// first when lg is odd, radix-4 passes after it.  Output lands in natural
// order in one of the two ping-pong buffers, which the call returns.
// Twiddles come from a per-length table tw[t] = exp(-2 pi i t / L) built in
// FP64 on the host; the inverse uses their conjugates.  No normalisation is
// applied in either direction.
#pragma once
#include <cuda_runtime.h>

namespace huv_dev {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <int DIR>
__device__ __forceinline__ float2 rot90(float2 a) {
  return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <int DIR>
__device__ __forceinline__ float2 tw_at(const float2* __restrict__ tw, int idx) {
  float2 w = __ldg(tw + idx);
  if (DIR > 0) w.y = -w.y;
  return w;
}

// DIR = -1 forward (e^{-2 pi i}), +1 inverse (e^{+2 pi i}).
template <int DIR>
__device__ float2* block_fft(float2* src, float2* dst, int lg, int S, const float2* __restrict__ tw) {
  const int L = 1 << lg;
  int Ns = 1;
  if (lg & 1) {
    const int half = L >> 1;
    const int total = S * half;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int s = t >> (lg - 1), j = t & (half - 1);
      const float2* in = src + (s << lg);
      float2* out = dst + (s << lg);
      const float2 v0 = in[j], v1 = in[j + half];
      out[2 * j] = cadd(v0, v1);
      out[2 * j + 1] = csub(v0, v1);
    }
    __syncthreads();
    float2* t = src;
    src = dst;
    dst = t;
    Ns = 2;
  }
  const int q = L >> 2;
  while (Ns < L) {
    const int total = S * q;
    const int tstep = L / (Ns * 4);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int s = t >> (lg - 2), j = t & (q - 1);
      const float2* in = src + (s << lg);
      float2* out = dst + (s << lg);
      const int k = j & (Ns - 1);
      float2 v0 = in[j], v1 = in[j + q], v2 = in[j + 2 * q], v3 = in[j + 3 * q];
      if (Ns > 1) {
        const int e = tstep * k;
        v1 = cmul(v1, tw_at<DIR>(tw, e));
        v2 = cmul(v2, tw_at<DIR>(tw, 2 * e));
        v3 = cmul(v3, tw_at<DIR>(tw, 3 * e));
      }
      const float2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
      const float2 b0 = cadd(v1, v3), b1 = rot90<DIR>(csub(v1, v3));
      const int base = ((j - k) << 2) + k;
      out[base] = cadd(a0, b0);
      out[base + Ns] = cadd(a1, b1);
      out[base + 2 * Ns] = csub(a0, b0);
      out[base + 3 * Ns] = csub(a1, b1);
    }
    __syncthreads();
    float2* t = src;
    src = dst;
    dst = t;
    Ns <<= 2;
  }
  return src;
}

// Largest power of two <= want whose `per_unit` bytes times it fit in the
// dynamic shared-memory budget of the FFT kernels (192 KiB).
inline int fit_units(int want, size_t per_unit) {
  const size_t budget = size_t(192) << 10;
  int u = 1;
  while (u * 2 <= want && static_cast<size_t>(u * 2) * per_unit <= budget) u *= 2;
  return u;
}

}  // namespace huv_dev
