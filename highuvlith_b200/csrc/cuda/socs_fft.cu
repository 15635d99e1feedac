// Plain FP32 FFT form of the SOCS aerial image, for sm_100a.
//
//   band_rows_fwd   : mask raster rows -> FFT along x -> keep orders [-hb, hb]
//   band_cols_fwd   : band columns -> FFT along y -> keep [-hb, hb]^2, optional
//                     pixel transfer, and the flare mean from the band
//   socs_rows_inv   : per (kernel k, band row my): K_k(my, .) . M(my, .) ->
//                     zero-padded inverse FFT along x on the evaluation grid
//   socs_cols_inv   : per strip of columns: inverse FFT along y of every
//                     kernel's band column, lambda-weighted |E|^2 summed over k
//                     in shared memory, normalisation + flare epilogue
//
// This is the device form of socs_intensity + normalize + apply_flare
// (crates/highuvlith-core/src/aerial.rs:1682-1748) fed by Mask::spectrum's
// raster path (mask.rs:630-635) or compute_from_transmittance's FFT
// (aerial.rs:1789-1798).  Kernel values arrive pre-scaled by
// sqrt(lambda_k / divisor) / N^2, so |E|^2 sums directly to the normalised
// image.  The flare mean is computed exactly from the band by Parseval:
// mean(I0) = sum_f W(f) |M(f)|^2 with W = sum_k lambda_k |u_k|^2 / N^4.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft_block.cuh"
#include "fft_reg.cuh"

namespace huv_dev {

// ------------------------------------------------------------ raster load
template <int KIND>
__device__ __forceinline__ float2 load_px(const void* base, size_t idx);
template <>
__device__ __forceinline__ float2 load_px<0>(const void* base, size_t idx) {
  return make_float2(static_cast<float>(static_cast<const uint8_t*>(base)[idx]), 0.f);
}
template <>
__device__ __forceinline__ float2 load_px<1>(const void* base, size_t idx) {
  return make_float2(static_cast<const float*>(base)[idx], 0.f);
}
template <>
__device__ __forceinline__ float2 load_px<2>(const void* base, size_t idx) {
  return static_cast<const float2*>(base)[idx];
}

// Forward FFT of raster rows, band [-hb, hb] kept.  Real inputs (KIND 0, 1)
// pack rows (2s, 2s+1) into one complex sequence and split the spectra;
// complex input (KIND 2) transforms one row per sequence.
// grid: (n / rows_per_block, clips); X: [clip][y][B], B = 2 hb + 1.
template <int KIND>
__global__ void band_rows_fwd(const void* __restrict__ in, int lg, int rows_per_block, int hb,
                              float2* __restrict__ X, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int row0 = blockIdx.x * rows_per_block;
  const bool real_in = KIND != 2;
  const int S = real_in ? rows_per_block / 2 : rows_per_block;
  float2* a = smem;
  float2* b = smem + (S << lg);
  const size_t plane = static_cast<size_t>(L) * L;
  const size_t cbase = static_cast<size_t>(clip) * plane;
  for (int t = threadIdx.x; t < (S << lg); t += blockDim.x) {
    const int s = t >> lg, i = t & (L - 1);
    if (real_in) {
      const float2 p = load_px<KIND>(in, cbase + static_cast<size_t>(row0 + 2 * s) * L + i);
      const float2 q = load_px<KIND>(in, cbase + static_cast<size_t>(row0 + 2 * s + 1) * L + i);
      a[t] = make_float2(p.x, q.x);
    } else {
      a[t] = load_px<KIND>(in, cbase + static_cast<size_t>(row0 + s) * L + i);
    }
  }
  __syncthreads();
  const float2* r = block_fft<-1>(a, b, lg, S, tw);
  const int outs = real_in ? 2 * S : S;
  for (int t = threadIdx.x; t < S * B; t += blockDim.x) {
    const int s = t / B, mi = t - s * B;
    const int m = mi - hb;
    const int idx = m & (L - 1);
    const float2 z = r[(s << lg) + idx];
    if (real_in) {
      const float2 zc = cconj(r[(s << lg) + ((L - idx) & (L - 1))]);
      const float2 xa = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y + zc.y));
      const float2 d = csub(z, zc);
      const float2 xb = make_float2(0.5f * d.y, -0.5f * d.x);
      const size_t ya = static_cast<size_t>(clip) * L + row0 + 2 * s;
      X[ya * B + mi] = xa;
      X[(ya + 1) * B + mi] = xb;
    } else {
      const size_t y = static_cast<size_t>(clip) * L + row0 + s;
      X[y * B + mi] = z;
    }
  }
  (void)outs;
}

// Forward FFT of the band columns along y; keeps [-hb, hb]^2, multiplies by
// the separable pixel transfer ptx (B floats; NULL = none) and, when W is
// given, writes this block's part of the flare mean sum_f W(f) |M(f)|^2 to
// parts[clip * gridDim.x + blockIdx.x] (summed in order by mean_reduce).
// grid: (ceil(B / cols_per_block), clips).
__global__ void band_cols_fwd(const float2* __restrict__ X, int lg, int hb, int cols_per_block,
                              const float* __restrict__ ptx, const float* __restrict__ W,
                              float2* __restrict__ Mband, float* __restrict__ parts,
                              const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  __shared__ float red[32];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int c0 = blockIdx.x * cols_per_block;
  const int nc = min(cols_per_block, B - c0);
  float2* a = smem;
  float2* b = smem + (cols_per_block << lg);
  const float2* Xc = X + static_cast<size_t>(clip) * L * B;
  float2* Mc = Mband + static_cast<size_t>(clip) * B * B;
  for (int t = threadIdx.x; t < (cols_per_block << lg); t += blockDim.x) {
    const int s = t & (cols_per_block - 1), y = t / cols_per_block;
    a[(s << lg) + y] = s < nc ? Xc[static_cast<size_t>(y) * B + c0 + s] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* r = block_fft<-1>(a, b, lg, cols_per_block, tw);
  float part = 0.f;
  for (int t = threadIdx.x; t < nc * B; t += blockDim.x) {
    const int s = t / B, mi = t - s * B;
    const int mx = c0 + s;
    const int idx = (mi - hb) & (L - 1);
    float2 v = r[(s << lg) + idx];
    if (ptx) {
      const float f = ptx[mi] * ptx[mx];
      v.x *= f;
      v.y *= f;
    }
    Mc[static_cast<size_t>(mi) * B + mx] = v;
    if (W) part += W[mi * B + mx] * (v.x * v.x + v.y * v.y);
  }
  if (parts) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      float sum = 0.f;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) sum += red[w];
      parts[static_cast<size_t>(clip) * gridDim.x + blockIdx.x] = sum;
    }
  }
}

// mean[clip] = sum of the clip's parts in index order (deterministic).
__global__ void mean_reduce(const float* __restrict__ parts, int nparts, int clips, float* __restrict__ mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= clips) return;
  float s = 0.f;
  for (int i = 0; i < nparts; ++i) s += parts[static_cast<size_t>(c) * nparts + i];
  mean[c] = s;
}

// Inverse transform along x of every (kernel, band row) product, on the
// evaluation grid of 2^lg points.  kband: [K][B][B] (pre-scaled); Mband:
// [clip][B][B]; T: [clip][K][B][Lg].  grid: (ceil(K*B / S), clips).
__global__ void socs_rows_inv(const float2* __restrict__ kband, float scale,
                              const float2* __restrict__ Mband, int K, int hb, int lg, int S,
                              float2* __restrict__ T, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int seq0 = blockIdx.x * S;
  const int nseq = min(S, K * B - seq0);
  float2* a = smem;
  float2* b = smem + (S << lg);
  for (int t = threadIdx.x; t < (S << lg); t += blockDim.x) a[t] = make_float2(0.f, 0.f);
  __syncthreads();
  const float2* Mc = Mband + static_cast<size_t>(clip) * B * B;
  for (int t = threadIdx.x; t < nseq * B; t += blockDim.x) {
    const int s = t / B, mx = t - s * B;
    const int seq = seq0 + s;
    const int k = seq / B, my = seq - k * B;
    const float2 m = Mc[static_cast<size_t>(my) * B + mx];
    const float2 u = kband ? kband[(static_cast<size_t>(k) * B + my) * B + mx] : make_float2(scale, 0.f);
    a[(s << lg) + ((mx - hb) & (L - 1))] = cmul(u, m);
  }
  __syncthreads();
  const float2* r = block_fft<+1>(a, b, lg, S, tw);
  float2* Tc = T + static_cast<size_t>(clip) * K * B * L;
  for (int t = threadIdx.x; t < (nseq << lg); t += blockDim.x) {
    const int s = t >> lg, x = t & (L - 1);
    Tc[(static_cast<size_t>(seq0 + s) << lg) + x] = r[t];
  }
}

// Column pass + accumulation.  MODE 0: out = keep * sum_k |E_k|^2 + flare * mean
// (mean per clip from band_cols_fwd).  MODE 1 (band interpolation): one
// "kernel" whose inverse transform is real; out = Re(E).
// grid: (Lg / Wc, clips); T as written by socs_rows_inv; out: [clip][Lg][Lg].
template <int MODE>
__global__ void socs_cols_inv(const float2* __restrict__ T, int K, int hb, int lg, int Wc,
                              float keep, float flare, const float* __restrict__ mean,
                              float* __restrict__ out, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int x0 = blockIdx.x * Wc;
  float2* a = smem;
  float2* b = smem + (Wc << lg);
  float* acc = reinterpret_cast<float*>(smem + 2 * (Wc << lg));  // [Wc][L]
  for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) acc[t] = 0.f;
  const float2* Tc = T + static_cast<size_t>(clip) * K * B * L;
  for (int k = 0; k < K; ++k) {
    for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) a[t] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int t = threadIdx.x; t < B * Wc; t += blockDim.x) {
      const int my = t / Wc, w = t - my * Wc;
      const float2 v = Tc[((static_cast<size_t>(k) * B + my) << lg) + x0 + w];
      a[(w << lg) + ((my - hb) & (L - 1))] = v;
    }
    __syncthreads();
    const float2* r = block_fft<+1>(a, b, lg, Wc, tw);
    for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) {
      const float2 e = r[t];
      if (MODE == 0)
        acc[t] += e.x * e.x + e.y * e.y;
      else
        acc[t] += e.x;
    }
    __syncthreads();
  }
  const float add = (MODE == 0 && mean) ? flare * mean[clip] : 0.f;
  const float mul = MODE == 0 ? keep : 1.f;
  float* oc = out + static_cast<size_t>(clip) * L * L;
  for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) {
    const int y = t / Wc, w = t - y * Wc;
    oc[static_cast<size_t>(y) * L + x0 + w] = mul * acc[(w << lg) + y] + add;
  }
}

// ------------------------------------------- register-radix (fft_reg.cuh)
// x-major band layout of the row transforms: Tt[clip][k][x][my], B values
// per x, so that the row kernel's stores and the column kernel's loads are
// both contiguous.  Used for L = 128 .. 1024 with 2 hb < L.

// Inverse transform along x of every (kernel, band row) product; S sequences
// per block.  grid: (ceil(K * B / S), clips).
// Six blocks per SM (40 registers) on the coarse grids, where a block's
// shared memory allows it (3.6 % faster at M = 160); the long transforms
// are held to three (their buffers allow three blocks at most).
template <int L, int S>
__global__ void __launch_bounds__(fr_threads(L, S), (L <= 256 ? 6 : 4))
    socs_rows_xt(const float2* __restrict__ kband, float scale, const float2* __restrict__ Mband, int K, int hb,
                 float2* __restrict__ Tt, const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  extern __shared__ float2 smem[];
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int seq0 = blockIdx.x * S;
  const int nseq = min(S, K * B - seq0);
  const int t = threadIdx.x;
  float2* P = smem;  // [S][B] band products
  float2* b0 = smem + S * B;
  const float2* Mc = Mband + static_cast<size_t>(clip) * B * B;
  // one warp per sequence: (k, my) once per row, lanes along mx (no divisions)
  for (int s = t >> 5; s < S; s += T / 32) {
    float2* Ps = P + s * B;
    if (s < nseq) {
      const int seq = seq0 + s;
      const int k = seq / B, my = seq - k * B;
      const float2* mrow = Mc + static_cast<size_t>(my) * B;
      const float2* urow = kband ? kband + (static_cast<size_t>(k) * B + my) * B : nullptr;
      for (int mx = t & 31; mx < B; mx += 32)
        Ps[mx] = cmul(urow ? urow[mx] : make_float2(scale, 0.f), mrow[mx]);
    } else {
      for (int mx = t & 31; mx < B; mx += 32) Ps[mx] = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  fr_first_pass_band<L, S, +1>(t, P, B, hb, b0);
  __syncthreads();
  const float2* src = b0;
  if constexpr (NP == 3) {
    fr_mid_pass_inplace<L, S, +1, 1>(t, b0, tw);
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
    if (t + b * T >= fr_nb(L, S, NP - 1)) break;
    int s, j;
    float2 v[R];
    fr_last_pass<L, S, +1>(t + b * T, src, tw, s, j, v);
    if (s >= nseq) continue;
    const int seq = seq0 + s;
    const int k = seq / B, my = seq - k * B;
    float2* o = Tt + (static_cast<size_t>(clip) * K + k) * L * B + my;
#pragma unroll
    for (int p = 0; p < R; ++p) o[static_cast<size_t>(j + p * (L / R)) * B] = v[p];
  }
}

// Column pass over Tt + accumulation, S sequences per block.  MODE 0: columns
// x0 + s; out = keep * sum_k |E_k|^2 + flare * mean, with the sum held in
// registers across k.  MODE 1 (band synthesis of a real image, K = 1): two
// columns per sequence, z = T(., x0 + 2s) + i T(., x0 + 2s + 1); each column
// is Hermitian in my, so Re and Im of the transform are the two real
// columns.  grid: (L / (S or 2 S), clips); out: [clip][L][L].  MODE 0 with
// `split` set writes v = I / interp_scale(mean) as two FP16 planes instead
// (hi, and lo = the rounding remainder), [clip][plane][L][L]: the B operand
// of the separable band interpolation on tensor cores.
// Three blocks per SM (80 registers) for the accumulating column pass at
// L = 160 (7.7 % faster than two; its 10 outputs per thread fit without
// spills); two elsewhere, where 12 or more outputs per thread would spill.
template <int L, int S, int MODE>
__global__ void __launch_bounds__(fr_threads(L, S), ((L == 160 && MODE == 0) || (L >= 384 && MODE == 1) ? 3 : 2))
    socs_cols_xt(const float2* __restrict__ Tt, int K, int hb, float keep, float flare,
                 const float* __restrict__ mean, float* __restrict__ out, const float2* __restrict__ tw,
                 __half* __restrict__ split) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  constexpr int XS = MODE == 1 ? 2 * S : S;
  static_assert(L % 2 == 0 && S % 2 == 0, "band blocks copied two elements (16 bytes) at a time");
  extern __shared__ float2 smem[];
  const int B = 2 * hb + 1;
  const int clip = blockIdx.y;
  const int x0 = blockIdx.x * XS;
  const int t = threadIdx.x;
  float2* P = smem;  // [S][B]
  float2* b0 = smem + S * B;
  constexpr int NO = fr_per(L, S, NP - 1) * R;  // outputs per thread
  float acc[NO];
  float2 res[NO];
#pragma unroll
  for (int i = 0; i < NO; ++i) {
    acc[i] = 0.f;
    res[i] = make_float2(0.f, 0.f);
  }
  // MODE 0: kernel k's band columns (one contiguous block of S B values)
  // arrive by cp.async in P[k & 1] while kernel k - 1 is transformed.
  float2* P2 = b0 + fr_buf(L, S);  // second band buffer (MODE 0), after the FFT buffer
  // The block is 16-byte aligned at both ends (L and S are even, so the
  // element offset ((clip K + k) L + x0) B and the length S B are even):
  // two elements per copy.
  auto prefetch = [&](int k) {
    const float2* src = Tt + ((static_cast<size_t>(clip) * K + k) * L + x0) * B;
    float2* dst = (k & 1) ? P2 : P;
    for (int e = 2 * t; e < S * B; e += 2 * T) fr_cp_async16(dst + e, src + e);
    fr_cp_commit();
  };
  if (MODE == 0) prefetch(0);
  float2 lw[fr_per(L, S, NP - 1)][R - 1];  // last-pass twiddles, the same for every kernel
  fr_last_twiddles<L, S, +1>(t, tw, lw);
  // first-pass input offsets into a kernel's band block, the same for every
  // kernel (MODE 0 loops over K kernels; MODE 1 has one)
  const bool pruned = MODE == 0 && 4 * hb < L;
  int boff[8];
  if (pruned) fr_band_offsets<L, S>(t, B, hb, boff);
  for (int k = 0; k < K; ++k) {
    const float2* Pk = P;
    if (MODE == 0) {
      if (k + 1 < K) {
        prefetch(k + 1);  // its buffer was last read by kernel k - 1's first pass, before that barrier
        fr_cp_wait<1>();
      } else {
        fr_cp_wait<0>();
      }
      Pk = (k & 1) ? P2 : P;
    } else {
      const float2* src = Tt + ((static_cast<size_t>(clip) * K + k) * L + x0) * B;
      for (int e = t; e < S * B; e += T) {
        const int s = e / B, my = e - s * B;
        const float2 a = src[static_cast<size_t>(2 * s) * B + my];
        const float2 c = src[static_cast<size_t>(2 * s + 1) * B + my];
        P[e] = make_float2(a.x - c.y, a.y + c.x);
      }
    }
    __syncthreads();
    if (pruned)
      fr_first_pass_band_off<L, S, +1>(t, Pk, boff, b0);
    else
      fr_first_pass_band<L, S, +1>(t, Pk, B, hb, b0);
    __syncthreads();
    const float2* cur = b0;
    if constexpr (NP == 3) {
      fr_mid_pass_inplace<L, S, +1, 1>(t, b0, tw);
      __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
      if (t + b * T >= fr_nb(L, S, NP - 1)) break;
      int s, j;
      float2 v[R];
      fr_last_pass_pre<L, S, +1>(t + b * T, cur, lw[b], s, j, v);
#pragma unroll
      for (int p = 0; p < R; ++p) {
        if (MODE == 0)
          acc[b * R + p] += v[p].x * v[p].x + v[p].y * v[p].y;
        else
          res[b * R + p] = v[p];
      }
    }
    // No barrier here: the next kernel's band buffer is written by cp.async
    // (MODE 0) or plain stores (MODE 1) into a buffer whose readers (this
    // first pass) passed the barrier above, and its first pass writes b0 only
    // after the next loop-top barrier, which every thread reaches after its
    // own last pass here.
  }
  const float add = (MODE == 0 && mean) ? flare * mean[clip] : 0.f;
  const float inv = (MODE == 0 && split) ? 1.f / interp_scale(mean ? mean[clip] : 0.f) : 1.f;
  float* oc = out + static_cast<size_t>(clip) * L * L;
#pragma unroll
  for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
    const int u = t + b * T;
    if (u >= fr_nb(L, S, NP - 1)) break;
    const int s = u % S, j = u / S;
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const size_t y = static_cast<size_t>(j + p * (L / R));
      if (MODE == 0 && split) {
        const float v = (keep * acc[b * R + p] + add) * inv;
        const __half hi = __float2half_rn(v);
        __half* sc = split + static_cast<size_t>(clip) * 2 * L * L + y * L + x0 + s;
        sc[0] = hi;
        sc[static_cast<size_t>(L) * L] = __float2half_rn(v - __half2float(hi));
      } else if (MODE == 0)
        oc[y * L + x0 + s] = keep * acc[b * R + p] + add;
      else
        *reinterpret_cast<float2*>(oc + y * L + x0 + 2 * s) = res[b * R + p];
    }
  }
}

// band_rows_fwd<1> (f32 rasters) with register-radix passes: S complex
// sequences per block, sequence s packing rows (2s, 2s+1) as re / im; the
// last pass leaves the spectra in natural order in shared memory, and the
// two real rows' bands are split from Z(m) and conj Z(-m).  The rows are
// real, X(y, -m) = conj X(y, m), so X holds the orders m = 0..hb alone.
// grid: (clips * L / (2 S)); X: [clip][y][hb + 1].
template <int L, int S, typename In = float>
__global__ void __launch_bounds__(fr_threads(L, S), (L >= 384 ? 4 : 1))
    band_rows_reg(const In* __restrict__ in, int hb, float2* __restrict__ X, const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  extern __shared__ float2 smem[];
  const size_t row0 = static_cast<size_t>(blockIdx.x) * 2 * S;
  const int t = threadIdx.x;
  float2* b0 = smem;
  if (t < fr_nb(L, S, 0)) {
    const int s = t % S, j = t / S;
    const In* ra = in + (row0 + 2 * s) * L + j;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r)
      v[r] = make_float2(static_cast<float>(ra[r * (L / 16)]), static_cast<float>(ra[L + r * (L / 16)]));
    fr_first_pass_vals<L, S, -1>(t, v, b0);
  }
  __syncthreads();
  float2* cur = b0;
  fr_mid_pass_inplace<L, S, -1, 1>(t, b0, tw);
  if constexpr (NP == 3) {
    __syncthreads();
    fr_mid_pass_inplace<L, S, -1, 2>(t, b0, tw);
  }
  __syncthreads();
  const int H = hb + 1;
  for (int e = t; e < S * H; e += T) {
    const int s = e / H, m = e - s * H;
    const float2 z = cur[fr_idx<S>(m, s)];
    const float2 zc = cconj(cur[fr_idx<S>(m == 0 ? 0 : L - m, s)]);
    const float2 xa = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y + zc.y));
    const float2 d = csub(z, zc);
    const float2 xb = make_float2(0.5f * d.y, -0.5f * d.x);
    X[(row0 + 2 * s) * H + m] = xa;
    X[(row0 + 2 * s + 1) * H + m] = xb;
  }
}

// band_cols_fwd with register-radix passes: forward FFT along y of S band
// columns per block, the first pass reading X directly.  X is [clip][y][B]
// (every order mx = -hb..hb), or, with `half`, the orders mx = 0..hb of a
// real raster alone, [clip][y][hb + 1] or (`transposed`) [clip][hb + 1][y]:
// the band of a real raster is Hermitian, M(-my, -mx) = conj M(my, mx), so
// the columns mx > 0 also give the columns -mx.  grid: (ceil(columns / S),
// clips).
template <int L, int S>
__global__ void __launch_bounds__(fr_threads(L, S))
    band_cols_reg(const float2* __restrict__ X, bool half, bool transposed, int hb, const float* __restrict__ ptx,
                  const float* __restrict__ W, float2* __restrict__ Mband, float* __restrict__ parts,
                  const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  extern __shared__ float2 smem[];
  __shared__ float red[T / 32];
  const int B = 2 * hb + 1;
  const int NC = half ? hb + 1 : B;  // columns held in X
  const int clip = blockIdx.y;
  const int c0 = blockIdx.x * S;
  const int t = threadIdx.x;
  float2* b0 = smem;
  const float2* Xc = X + static_cast<size_t>(clip) * L * NC;
  if (t < fr_nb(L, S, 0)) {
    const int s = t % S, j = t / S;
    const bool live = c0 + s < NC;
    float2 v[16];
    const size_t col_base = transposed ? static_cast<size_t>(c0 + s) * L : static_cast<size_t>(c0 + s);
    const size_t row_step = transposed ? 1 : static_cast<size_t>(NC);
#pragma unroll
    for (int r = 0; r < 16; ++r)
      v[r] = live ? Xc[col_base + static_cast<size_t>(j + r * (L / 16)) * row_step] : make_float2(0.f, 0.f);
    fr_first_pass_vals<L, S, -1>(t, v, b0);
  }
  __syncthreads();
  const float2* cur = b0;
  if constexpr (NP == 3) {
    // one buffer: more blocks per SM to keep the column loads in flight
    fr_mid_pass_inplace<L, S, -1, 1>(t, b0, tw);
    __syncthreads();
  }
  float2* Mc = Mband + static_cast<size_t>(clip) * B * B;
  float part = 0.f;
#pragma unroll
  for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
    if (t + b * T >= fr_nb(L, S, NP - 1)) break;
    // butterfly (s, j) produces orders j + p L / R: skip it unless one of
    // them lies in the band (75 of 256 last-pass butterflies at L = 1024, h = 37)
    {
      const int u = t + b * T, su = u % S, ju = u / S;
      bool need = false;
#pragma unroll
      for (int p = 0; p < R; ++p) {
        const int idx = ju + p * (L / R);
        need = need || idx <= hb || idx >= L - hb;
      }
      if (!need || c0 + su >= NC) continue;
    }
    int s, j;
    float2 v[R];
    fr_last_pass<L, S, -1>(t + b * T, cur, tw, s, j, v);
    const int mx = half ? hb + c0 + s : c0 + s;
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const int idx = j + p * (L / R);
      const int mi = idx <= hb ? idx + hb : (idx >= L - hb ? idx - L + hb : -1);
      if (mi < 0) continue;
      float2 val = v[p];
      if (ptx) {
        const float f = ptx[mi] * ptx[mx];
        val.x *= f;
        val.y *= f;
      }
      Mc[static_cast<size_t>(mi) * B + mx] = val;
      if (W) part += W[mi * B + mx] * (val.x * val.x + val.y * val.y);
      if (half && mx > hb) {
        // the mirrored order (-my, -mx)
        const int mi2 = 2 * hb - mi, mx2 = 2 * hb - mx;
        float2 w2 = cconj(v[p]);
        if (ptx) {
          const float f = ptx[mi2] * ptx[mx2];
          w2.x *= f;
          w2.y *= f;
        }
        Mc[static_cast<size_t>(mi2) * B + mx2] = w2;
        if (W) part += W[mi2 * B + mx2] * (w2.x * w2.x + w2.y * w2.y);
      }
    }
  }
  if (parts) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((t & 31) == 0) red[t >> 5] = part;
    __syncthreads();
    if (t == 0) {
      float sum = 0.f;
      for (int w = 0; w < T / 32; ++w) sum += red[w];
      parts[static_cast<size_t>(clip) * gridDim.x + blockIdx.x] = sum;
    }
  }
}

}  // namespace huv_dev

// ------------------------------------------------------------ launchers
namespace huv_launch {

using namespace huv_dev;

static int pick_threads(int work) { return work >= 256 ? 256 : 128; }

cudaError_t mask_rows_tc(const void* in, int n, int hb, int clips, float2* X, const uint8_t* digits, int* err,
                         cudaStream_t st, bool transposed);
bool xt_ok(int lg, int hb);
cudaError_t socs_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int lgm, int clips,
                      float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols(const float2* T, int K, int hb, int lgm, int clips, float keep, float flare,
                      const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);

// Mask (or image) band: rows then columns.  When W is given, `mean` must hold
// clips + clips * ceil(B / 4) floats: the first `clips` receive the flare
// means, the rest holds the per-block parts.  `row_digits` (may be NULL) is
// the device digit table of the tensor-core row band for u8 rasters; `err`
// receives that kernel's timeout code.
cudaError_t band_forward(const void* in, int kind, int n, int lg, int hb, int clips, float2* X,
                         float2* Mband, const float* ptx, const float* W, float* mean,
                         const float2* tw, cudaStream_t st, const uint8_t* row_digits, int* err) {
  // n need not be a power of two when the register-radix kernels serve it
  // (160 = 16 x 10, 192 = 16 x 12); the radix-4 kernels use lg = log2 n.
  const bool pow2 = (n & (n - 1)) == 0;
  const int S = pow2 ? fit_units(2, 2 * (sizeof(float2) << lg)) : 1;
  const int rows_per_block = (kind == 2) ? S : 2 * S;
  const size_t sm1 = 2 * (static_cast<size_t>(S) << lg) * sizeof(float2);
  dim3 g1(n / rows_per_block, clips);
  const int th = pick_threads(S << (lg - 2));
  // u8 rasters take the exact integer tensor-core row band when the shape
  // and the input's alignment allow it; f32 rasters of 1024-point rows the
  // register-radix rows (4 sequences per block read 32-byte row segments;
  // with more, shorter rows per block the radix-4 kernel's coalesced loads
  // win).
  cudaError_t rows_tc = cudaErrorNotSupported;
  // the register-radix columns read a transposed row band ([clip][m][y]) when
  // the tensor-core rows produce it
  const bool cols_reg = xt_ok(n, hb);
  // (and then, as the register-radix rows do, only the orders m = 0..hb of
  // the real rasters: `half`)
  bool x_transposed = false, half = false;
  if (kind == 0 && row_digits) {
    rows_tc = mask_rows_tc(in, n, hb, clips, X, row_digits, err, st, cols_reg);
    x_transposed = half = rows_tc == cudaSuccess && cols_reg;
    if (rows_tc != cudaSuccess && rows_tc != cudaErrorNotSupported) return rows_tc;
  }
  if (kind == 1 && (n == 1024 || n == 160 || n == 192 || n == 384 || n == 2048) && xt_ok(n, hb)) {
    const int Sr = xt_S(n);
    const dim3 gr(static_cast<unsigned>(static_cast<size_t>(clips) * n / (2 * Sr)));
    const size_t smr = static_cast<size_t>(fr_buf(n, Sr)) * sizeof(float2);
    const float* fin = static_cast<const float*>(in);
    if (n == 1024)
      band_rows_reg<1024, 4><<<gr, 256, smr, st>>>(fin, hb, X, tw);
    else if (n == 2048)
      band_rows_reg<2048, 2><<<gr, 256, smr, st>>>(fin, hb, X, tw);
    else if (n == 384)
      band_rows_reg<384, 8><<<gr, 256, smr, st>>>(fin, hb, X, tw);
    else if (n == 160)
      band_rows_reg<160, 16><<<gr, 256, smr, st>>>(fin, hb, X, tw);
    else
      band_rows_reg<192, 16><<<gr, 256, smr, st>>>(fin, hb, X, tw);
    rows_tc = cudaSuccess;
    half = true;
  }
  // u8 rows of 2048 points whose band is too wide for the tensor-core rows
  // (3 digit-plane accumulators past 512 TMEM columns): register-radix rows
  if (kind == 0 && rows_tc != cudaSuccess && n == 2048 && xt_ok(n, hb)) {
    const int Sr = xt_S(n);
    const dim3 gr(static_cast<unsigned>(static_cast<size_t>(clips) * n / (2 * Sr)));
    const size_t smr = static_cast<size_t>(fr_buf(n, Sr)) * sizeof(float2);
    band_rows_reg<2048, 2, uint8_t><<<gr, 256, smr, st>>>(static_cast<const uint8_t*>(in), hb, X, tw);
    rows_tc = cudaSuccess;
    half = true;
  }
  if (!pow2 && rows_tc != cudaSuccess) return cudaErrorInvalidValue;  // no radix-4 kernel for this length
  // Only device rasters come here (rectangle clips take the analytic path).
  switch (kind) {
    case 0:
      if (rows_tc != cudaSuccess) band_rows_fwd<0><<<g1, th, sm1, st>>>(in, lg, rows_per_block, hb, X, tw);
      break;
    case 1:
      if (rows_tc != cudaSuccess) band_rows_fwd<1><<<g1, th, sm1, st>>>(in, lg, rows_per_block, hb, X, tw);
      break;
    case 2: band_rows_fwd<2><<<g1, th, sm1, st>>>(in, lg, rows_per_block, hb, X, tw); break;
    default: return cudaErrorInvalidValue;
  }
  const int B = 2 * hb + 1;
  float* parts = (W && mean) ? mean + clips : nullptr;
  int nblk;
  if (cols_reg) {
    // register-radix columns: S <= 4 ... 32 columns per block, at most
    // ceil(B / 4) parts per clip as the callers size them
    const int S = xt_S(n);
    nblk = ((half ? hb + 1 : B) + S - 1) / S;
    const dim3 g(nblk, clips);
    const size_t sm = xt_buf_bytes(n);
    switch (n) {
      case 128: band_cols_reg<128, 32><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 160: band_cols_reg<160, 16><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 192: band_cols_reg<192, 16><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 256: band_cols_reg<256, 16><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 384: band_cols_reg<384, 8><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 512: band_cols_reg<512, 8><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 2048: band_cols_reg<2048, 2><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      case 1024: band_cols_reg<1024, 4><<<g, 256, sm, st>>>(X, half, x_transposed, hb, ptx, W, Mband, parts, tw); break;
      default: return cudaErrorInvalidValue;
    }
  } else {
    if (!pow2) return cudaErrorInvalidValue;
    const int cpb = fit_units(4, 2 * (sizeof(float2) << lg));
    nblk = (B + cpb - 1) / cpb;
    const size_t sm2 = 2 * (static_cast<size_t>(cpb) << lg) * sizeof(float2);
    band_cols_fwd<<<dim3(nblk, clips), 256, sm2, st>>>(X, lg, hb, cpb, ptx, W, Mband, parts, tw);
  }
  if (parts) mean_reduce<<<(clips + 127) / 128, 128, 0, st>>>(parts, nblk, clips, mean);
  return cudaGetLastError();
}

// Whether the register-radix kernels (x-major band layout) apply to length
// L (128, 160, 192, 256, 512, 1024, 2048) and band half-width hb: every one of
// them within the shared-memory budget.
bool xt_ok(int L, int hb) {
  const int S = xt_S(L);
  if (S == 0 || 2 * hb >= L) return false;
  // the largest user: the column pass with two band buffers and two FFT buffers
  const size_t cols = 2 * static_cast<size_t>(S) * (2 * hb + 1) * sizeof(float2) +
                      2 * static_cast<size_t>(fr_buf(L, S)) * sizeof(float2);
  return cols <= static_cast<size_t>(kXtSmemMax);
}

static int ilog2_exact(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return (1 << l) == v ? l : -1;
}

// Rows of every (kernel, band row) product into T on a grid of L points,
// x-major when xt_ok (the layout socs_cols_x reads), else (L a power of two)
// the [k][my][x] layout of socs_rows.
cudaError_t socs_rows_x(const float2* kband, float scale, const float2* Mband, int K, int hb, int L, int clips,
                        float2* T, const float2* tw, cudaStream_t st) {
  if (!xt_ok(L, hb)) {
    const int lg = ilog2_exact(L);
    if (lg < 0) return cudaErrorInvalidValue;
    return socs_rows(kband, scale, Mband, K, hb, lg, clips, T, tw, st);
  }
  const int B = 2 * hb + 1, S = xt_S(L);
  const dim3 g((K * B + S - 1) / S, clips);
  const size_t sm = static_cast<size_t>(S) * B * sizeof(float2) + xt_buf_bytes(L);
  switch (L) {
    case 128: socs_rows_xt<128, 32><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 160: socs_rows_xt<160, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 192: socs_rows_xt<192, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 256: socs_rows_xt<256, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 384: socs_rows_xt<384, 8><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 512: socs_rows_xt<512, 8><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 2048: socs_rows_xt<2048, 2><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    case 1024: socs_rows_xt<1024, 4><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, T, tw); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

namespace {
cudaError_t cols_xt(const float2* T, int K, int hb, int L, int clips, float keep, float flare, const float* mean,
                    float* out, int mode, const float2* tw, cudaStream_t st, __half* split) {
  const int B = 2 * hb + 1, S = xt_S(L);
  // band columns (mode 0: double-buffered) and the one FFT buffer
  const size_t sm = static_cast<size_t>(S) * B * sizeof(float2) * (mode == 0 ? 2 : 1) + xt_buf_bytes(L);
  const dim3 g(L / (mode == 0 ? S : 2 * S), clips);
#define HUV_COLS_XT(LL, SS)                                                                                   \
  if (mode == 0)                                                                                            \
    socs_cols_xt<LL, SS, 0><<<g, 256, sm, st>>>(T, K, hb, keep, flare, mean, out, tw, split);               \
  else                                                                                                      \
    socs_cols_xt<LL, SS, 1><<<g, 256, sm, st>>>(T, K, hb, keep, flare, mean, out, tw, nullptr);
  switch (L) {
    case 128: HUV_COLS_XT(128, 32) break;
    case 160: HUV_COLS_XT(160, 16) break;
    case 192: HUV_COLS_XT(192, 16) break;
    case 256: HUV_COLS_XT(256, 16) break;
    case 384: HUV_COLS_XT(384, 8) break;
    case 512: HUV_COLS_XT(512, 8) break;
    case 2048: HUV_COLS_XT(2048, 2) break;
    case 1024: HUV_COLS_XT(1024, 4) break;
    default: return cudaErrorInvalidValue;
  }
#undef HUV_COLS_XT
  return cudaGetLastError();
}
}  // namespace

// Column pass over socs_rows_x's T (same lgm and hb).  mode 0: sum of |E_k|^2;
// mode 1: synthesis of a real image from a Hermitian band (K = 1), two
// columns per transform when xt_ok.
cudaError_t socs_cols_x(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                        const float* mean, float* out, int mode, const float2* tw, cudaStream_t st) {
  if (!xt_ok(L, hb)) {
    const int lg = ilog2_exact(L);
    if (lg < 0) return cudaErrorInvalidValue;
    return socs_cols(T, K, hb, lg, clips, keep, flare, mean, out, mode, tw, st);
  }
  return cols_xt(T, K, hb, L, clips, keep, flare, mean, out, mode, tw, st, nullptr);
}

// socs_cols_x mode 0 writing (keep * sum |E_k|^2 + flare * mean) / s, s =
// interp_scale(mean), as split FP16 planes [clip][2][L][L] (half elements at
// `split`).  Needs xt_ok(L, hb) and the per-clip mean.
cudaError_t socs_cols_split(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                            const float* mean, void* split, const float2* tw, cudaStream_t st) {
  if (!xt_ok(L, hb) || !mean) return cudaErrorInvalidValue;
  return cols_xt(T, K, hb, L, clips, keep, flare, mean, nullptr, 0, tw, st, static_cast<__half*>(split));
}

cudaError_t socs_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int lgm, int clips,
                      float2* T, const float2* tw, cudaStream_t st) {
  const int B = 2 * hb + 1;
  const int S = fit_units(4, 2 * (sizeof(float2) << lgm));
  const size_t sm3 = 2 * (static_cast<size_t>(S) << lgm) * sizeof(float2);
  dim3 g3((K * B + S - 1) / S, clips);
  socs_rows_inv<<<g3, 256, sm3, st>>>(kband, scale, Mband, K, hb, lgm, S, T, tw);
  return cudaGetLastError();
}

cudaError_t socs_cols(const float2* T, int K, int hb, int lgm, int clips, float keep, float flare,
                      const float* mean, float* out, int mode, const float2* tw, cudaStream_t st) {
  const int L = 1 << lgm;
  const int Wc = std::min(L, fit_units(8, 2 * (sizeof(float2) << lgm) + (sizeof(float) << lgm)));
  const size_t sm4 = (2 * (static_cast<size_t>(Wc) << lgm)) * sizeof(float2) +
                     (static_cast<size_t>(Wc) << lgm) * sizeof(float);
  dim3 g4(L / Wc, clips);
  if (mode == 0)
    socs_cols_inv<0><<<g4, 256, sm4, st>>>(T, K, hb, lgm, Wc, keep, flare, mean, out, tw);
  else
    socs_cols_inv<1><<<g4, 256, sm4, st>>>(T, K, hb, lgm, Wc, keep, flare, mean, out, tw);
  return cudaGetLastError();
}

cudaError_t field_fused_set_smem();

cudaError_t set_smem_limits() {
  const int big = 200 * 1024;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(band_rows_fwd<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(band_rows_fwd<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(band_rows_fwd<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(band_cols_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(socs_rows_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(socs_cols_inv<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(socs_cols_inv<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  const int xt = kXtSmemMax;
#define HUV_XT_ATTR(K)                                                                    \
  if ((e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, xt))) return e;
#define HUV_XT_ALL(LL, SS)                                                                                \
  HUV_XT_ATTR((socs_rows_xt<LL, SS>)) HUV_XT_ATTR((socs_cols_xt<LL, SS, 0>))                           \
  HUV_XT_ATTR((socs_cols_xt<LL, SS, 1>)) HUV_XT_ATTR((band_cols_reg<LL, SS>))
  HUV_XT_ALL(128, 32) HUV_XT_ALL(160, 16) HUV_XT_ALL(192, 16) HUV_XT_ALL(256, 16) HUV_XT_ALL(384, 8) HUV_XT_ALL(512, 8)
  HUV_XT_ALL(1024, 4) HUV_XT_ALL(2048, 2)
  HUV_XT_ATTR((band_rows_reg<1024, 4>)) HUV_XT_ATTR((band_rows_reg<160, 16>))
  HUV_XT_ATTR((band_rows_reg<192, 16>)) HUV_XT_ATTR((band_rows_reg<2048, 2>)) HUV_XT_ATTR((band_rows_reg<384, 8>))
  HUV_XT_ATTR((band_rows_reg<2048, 2, uint8_t>))
#undef HUV_XT_ALL
#undef HUV_XT_ATTR
  return field_fused_set_smem();
}

}  // namespace huv_launch
