// Fourier-neural-operator surrogate of the SOCS image: inference, training
// (forward + backward + Adam) and the input gradient used inside ILT.
//
// Network (channels-last activations, BF16 storage, FP32 arithmetic):
//   v0 = Lift(a, x/S, y/S)                                    3 -> C
//   z_l = SpecConv_l(v_l) + W_l v_l + b_l,  v_{l+1} = GELU(z_l) (l < L-1), v_L = z_{L-1}
//   out = Q2 . GELU(Q1 v_L + b1) + b2                          C -> P -> 1
//   SpecConv(v)(p) = S^-2 Re sum_{ky, kx < m} w_kx Y(ky, kx) e^{+2 pi i (ky y + kx x)/S},
//   Y(ky, kx, o) = sum_i X(ky, kx, i) R(ky, kx, i, o),  X = DFT(v) at the retained
//   modes (kx in [0, m), ky in [0, m) U [S - m, S)), w_0 = 1, w_kx = 2.
// The DFTs over the retained modes are direct sums with FP64-built twiddle
// tables (the mode count is small next to S).  Weight gradients are reduced
// per block and added with atomics.  There is no counterpart in the reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../../include/huv_b200.h"
#include "../engine.hpp"

namespace huv_dev {

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}
__device__ __forceinline__ float ld(const __nv_bfloat16* p, size_t i) { return __bfloat162float(p[i]); }
__device__ __forceinline__ float ld(const float* p, size_t i) { return p[i]; }

// ------------------------------------------------------------ lift
// v0[b][p][c] = Wl[c][0] a + Wl[c][1] x/S + Wl[c][2] y/S + bl[c]
__global__ void fno_lift(const float* __restrict__ a, int S, int C, const float* __restrict__ Wl,
                         const float* __restrict__ bl, __nv_bfloat16* __restrict__ v, size_t total) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t % C);
    const size_t bp = t / C;
    const int p = static_cast<int>(bp % (static_cast<size_t>(S) * S));
    const float gx = static_cast<float>(p % S) / S, gy = static_cast<float>(p / S) / S;
    v[t] = __float2bfloat16_rn(Wl[c * 3] * a[bp] + Wl[c * 3 + 1] * gx + Wl[c * 3 + 2] * gy + bl[c]);
  }
}

// ------------------------------------------------------------ DFT along x
// out[b][y][kx][c] (complex) = sum_x in[b][y][x][c] e^{-2 pi i kx x / S}, kx < m.
// grid: (S, B); block: C * ceil(...) threads, each (kx, c) pair strided.
template <typename T>
__global__ void fno_dft_x(const T* __restrict__ in, int S, int C, int m, const float2* __restrict__ twx,
                          float2* __restrict__ out) {
  extern __shared__ float srow[];  // [S][C]
  const int y = blockIdx.x, b = blockIdx.y;
  const size_t row = (static_cast<size_t>(b) * S + y) * S * C;
  for (int t = threadIdx.x; t < S * C; t += blockDim.x) srow[t] = ld(in, row + t);
  __syncthreads();
  for (int t = threadIdx.x; t < m * C; t += blockDim.x) {
    const int kx = t / C, c = t - kx * C;
    float re = 0.f, im = 0.f;
    const float2* tw = twx + static_cast<size_t>(kx) * S;  // e^{-2 pi i kx x / S}
    for (int x = 0; x < S; ++x) {
      const float v = srow[x * C + c];
      const float2 w = __ldg(tw + x);
      re += v * w.x;
      im += v * w.y;
    }
    out[((static_cast<size_t>(b) * S + y) * m + kx) * C + c] = make_float2(re, im);
  }
}

// ------------------------------------------------------------ DFT along y
// Forward (to modes): out[b][j][kx][c] = sum_y in[b][y][kx][c] e^{-2 pi i ky_j y / S}.
// Inverse (from modes): out[b][y][kx][c] = sum_j in[b][j][kx][c] e^{+2 pi i ky_j y / S}.
// twy[j][y] = e^{-2 pi i ky_j y / S}; grid: (rows_out, B).
template <bool INVERSE>
__global__ void fno_dft_y(const float2* __restrict__ in, int S, int C, int m, const float2* __restrict__ twy,
                          float2* __restrict__ out) {
  const int r = blockIdx.x, b = blockIdx.y;
  const int J = 2 * m;
  const int rows_in = INVERSE ? J : S;
  const int rows_out = INVERSE ? S : J;
  (void)rows_out;
  for (int t = threadIdx.x; t < m * C; t += blockDim.x) {
    float re = 0.f, im = 0.f;
    for (int q = 0; q < rows_in; ++q) {
      const float2 v = in[((static_cast<size_t>(b) * rows_in + q) * m) * C + t];
      float2 w = INVERSE ? __ldg(twy + static_cast<size_t>(q) * S + r) : __ldg(twy + static_cast<size_t>(r) * S + q);
      if (INVERSE) w.y = -w.y;
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
    }
    out[((static_cast<size_t>(b) * (INVERSE ? S : J) + r) * m) * C + t] = make_float2(re, im);
  }
}

// ------------------------------------------------------------ mode mixing
// Y[b][j][kx][o] = sum_i X[b][j][kx][i] R[j][kx][i][o]; grid: (J*m, B), block C.
__global__ void fno_mix(const float2* __restrict__ X, const float2* __restrict__ R, int C, int modes,
                        float2* __restrict__ Y) {
  extern __shared__ float2 sx[];
  const int md = blockIdx.x, b = blockIdx.y;
  const float2* xr = X + (static_cast<size_t>(b) * modes + md) * C;
  for (int t = threadIdx.x; t < C; t += blockDim.x) sx[t] = xr[t];
  __syncthreads();
  const float2* rr = R + static_cast<size_t>(md) * C * C;
  for (int o = threadIdx.x; o < C; o += blockDim.x) {
    float re = 0.f, im = 0.f;
    for (int i = 0; i < C; ++i) {
      const float2 x = sx[i], w = rr[i * C + o];
      re += x.x * w.x - x.y * w.y;
      im += x.x * w.y + x.y * w.x;
    }
    Y[(static_cast<size_t>(b) * modes + md) * C + o] = make_float2(re, im);
  }
}

// dX = sum_o dY conj(R); dR += conj(X) dY (summed over the batch).
__global__ void fno_mix_bwd(const float2* __restrict__ X, const float2* __restrict__ dY, const float2* __restrict__ R,
                            int C, int modes, int B, float2* __restrict__ dX, float2* __restrict__ dR) {
  extern __shared__ float2 sh[];  // [B][C] dY then [B][C] X
  const int md = blockIdx.x;
  float2* sdy = sh;
  float2* sxx = sh + B * C;
  for (int t = threadIdx.x; t < B * C; t += blockDim.x) {
    const int b = t / C, c = t - b * C;
    sdy[t] = dY[(static_cast<size_t>(b) * modes + md) * C + c];
    sxx[t] = X[(static_cast<size_t>(b) * modes + md) * C + c];
  }
  __syncthreads();
  const float2* rr = R + static_cast<size_t>(md) * C * C;
  float2* drr = dR + static_cast<size_t>(md) * C * C;
  for (int t = threadIdx.x; t < C * C; t += blockDim.x) {
    const int i = t / C, o = t - i * C;
    float re = 0.f, im = 0.f;
    for (int b = 0; b < B; ++b) {
      const float2 x = sxx[b * C + i], d = sdy[b * C + o];
      re += x.x * d.x + x.y * d.y;
      im += x.x * d.y - x.y * d.x;
    }
    drr[t].x += re;
    drr[t].y += im;
  }
  for (int t = threadIdx.x; t < B * C; t += blockDim.x) {
    const int b = t / C, i = t - b * C;
    float re = 0.f, im = 0.f;
    for (int o = 0; o < C; ++o) {
      const float2 d = sdy[b * C + o], w = rr[i * C + o];
      re += d.x * w.x + d.y * w.y;
      im += d.y * w.x - d.x * w.y;
    }
    dX[(static_cast<size_t>(b) * modes + md) * C + i] = make_float2(re, im);
  }
}

// ------------------------------------------------------------ layer output
// z = S^-2 Re sum_kx w_kx Z[y][kx][o] e^{+i th} + sum_i W[o][i] v[i] + b[o];
// v_next = GELU(z) (or z for the last layer).  grid: (S, B), block 256.
__global__ void fno_layer_out(const float2* __restrict__ Z, const __nv_bfloat16* __restrict__ v,
                              const float* __restrict__ W, const float* __restrict__ bias, int S, int C, int m,
                              const float2* __restrict__ twx, int act, __nv_bfloat16* __restrict__ zsave,
                              __nv_bfloat16* __restrict__ vnext) {
  extern __shared__ float sm[];
  float* sW = sm;                                           // [C][C]
  float2* sZ = reinterpret_cast<float2*>(sW + C * C);       // [m][C]
  const int y = blockIdx.x, b = blockIdx.y;
  for (int t = threadIdx.x; t < C * C; t += blockDim.x) sW[t] = W[t];
  const float2* Zr = Z + (static_cast<size_t>(b) * S + y) * m * C;
  const float inv = 1.f / (static_cast<float>(S) * S);
  for (int t = threadIdx.x; t < m * C; t += blockDim.x) {
    const float w = (t / C) == 0 ? inv : 2.f * inv;
    sZ[t] = make_float2(Zr[t].x * w, Zr[t].y * w);
  }
  __syncthreads();
  const size_t row = (static_cast<size_t>(b) * S + y) * S * C;
  for (int t = threadIdx.x; t < S * C; t += blockDim.x) {
    const int x = t / C, o = t - x * C;
    float acc = bias[o];
    for (int kx = 0; kx < m; ++kx) {
      const float2 w = __ldg(twx + static_cast<size_t>(kx) * S + x);  // e^{-i th}: use conj
      const float2 z = sZ[kx * C + o];
      acc += z.x * w.x + z.y * w.y;  // Re(z e^{+i th})
    }
    const __nv_bfloat16* vp = v + row + static_cast<size_t>(x) * C;
    const float* wr = sW + o * C;
    for (int i = 0; i < C; ++i) acc += wr[i] * __bfloat162float(vp[i]);
    zsave[row + t] = __float2bfloat16_rn(acc);
    vnext[row + t] = __float2bfloat16_rn(act ? gelu(acc) : acc);
  }
}

// Backward of the layer output: dz = dvnext * GELU'(z) (or dvnext); writes dz
// (f32), dv = W^T dz (f32, overwriting dv), dW += dz v^T, db += dz.
// grid: (S, B), block 256; the row is walked in tiles of 64 pixels with the
// weight-gradient partials in registers (C = 64: 16 (o, i) pairs per thread).
__global__ void __launch_bounds__(256) fno_layer_bwd(const float* __restrict__ dvnext,
                                                      const __nv_bfloat16* __restrict__ z,
                                                      const __nv_bfloat16* __restrict__ v,
                                                      const float* __restrict__ W, int S, int act,
                                                      float* __restrict__ dz, float* __restrict__ dv,
                                                      float* __restrict__ dW, float* __restrict__ db) {
  constexpr int C = 64, XT = 64;
  __shared__ float sW[C * C];
  __shared__ float sdz[XT * C];
  __shared__ float sv[XT * C];
  const int y = blockIdx.x, b = blockIdx.y;
  const size_t row = (static_cast<size_t>(b) * S + y) * S * C;
  for (int t = threadIdx.x; t < C * C; t += blockDim.x) sW[t] = W[t];
  float gw[16], gb = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) gw[q] = 0.f;
  const int xt = min(XT, S);  // S is a power of two, so xt divides S
  for (int x0 = 0; x0 < S; x0 += xt) {
    __syncthreads();
    for (int t = threadIdx.x; t < xt * C; t += blockDim.x) {
      const size_t g = row + static_cast<size_t>(x0) * C + t;
      const float gv = dvnext[g];
      const float d = act ? gv * gelu_grad(__bfloat162float(z[g])) : gv;
      sdz[t] = d;
      dz[g] = d;
      sv[t] = __bfloat162float(v[g]);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < xt * C; t += blockDim.x) {
      const int x = t / C, i = t - x * C;
      float acc = 0.f;
#pragma unroll 8
      for (int o = 0; o < C; ++o) acc += sW[o * C + i] * sdz[x * C + o];
      dv[row + static_cast<size_t>(x0) * C + t] = acc;
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int pr = threadIdx.x + q * 256;  // (o, i) pair
      const int o = pr / C, i = pr - o * C;
      float acc = 0.f;
      for (int x = 0; x < xt; ++x) acc += sdz[x * C + o] * sv[x * C + i];
      gw[q] += acc;
    }
    if (threadIdx.x < C)
      for (int x = 0; x < xt; ++x) gb += sdz[x * C + threadIdx.x];
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) atomicAdd(dW + threadIdx.x + q * 256, gw[q]);
  if (threadIdx.x < C) atomicAdd(db + threadIdx.x, gb);
}

// dv[b][y][x][c] += Re sum_kx Z[b][y][kx][c] e^{+2 pi i kx x / S}  (weight 1).
__global__ void fno_spec_to_dv(const float2* __restrict__ Z, int S, int C, int m, const float2* __restrict__ twx,
                               float* __restrict__ dv) {
  extern __shared__ float2 sZ[];
  const int y = blockIdx.x, b = blockIdx.y;
  const float2* Zr = Z + (static_cast<size_t>(b) * S + y) * m * C;
  for (int t = threadIdx.x; t < m * C; t += blockDim.x) sZ[t] = Zr[t];
  __syncthreads();
  const size_t row = (static_cast<size_t>(b) * S + y) * S * C;
  for (int t = threadIdx.x; t < S * C; t += blockDim.x) {
    const int x = t / C, c = t - x * C;
    float acc = 0.f;
    for (int kx = 0; kx < m; ++kx) {
      const float2 w = __ldg(twx + static_cast<size_t>(kx) * S + x);
      const float2 z = sZ[kx * C + c];
      acc += z.x * w.x + z.y * w.y;
    }
    dv[row + t] += acc;
  }
}

// Scale dY(j, kx) by w_kx / S^2 (the adjoint of the forward output weights).
__global__ void fno_scale_modes(float2* __restrict__ Y, int B, int J, int m, int C, float inv_s2) {
  const size_t total = static_cast<size_t>(B) * J * m * C;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int kx = static_cast<int>((t / C) % m);
    const float w = (kx == 0 ? 1.f : 2.f) * inv_s2;
    Y[t].x *= w;
    Y[t].y *= w;
  }
}

// ------------------------------------------------------------ projection
// out[b][p] = sum_j Q2[j] GELU(sum_c Q1[j][c] v[p][c] + b1[j]) + b2.
__global__ void fno_proj(const __nv_bfloat16* __restrict__ v, const float* __restrict__ Q1, const float* __restrict__ b1,
                         const float* __restrict__ Q2, const float* __restrict__ b2, int C, int P, size_t npix,
                         float* __restrict__ out) {
  extern __shared__ float sm[];
  float* sQ1 = sm;            // [P][C]
  float* sb1 = sQ1 + P * C;   // [P]
  float* sQ2 = sb1 + P;       // [P]
  for (int t = threadIdx.x; t < P * C; t += blockDim.x) sQ1[t] = Q1[t];
  for (int t = threadIdx.x; t < P; t += blockDim.x) {
    sb1[t] = b1[t];
    sQ2[t] = Q2[t];
  }
  __syncthreads();
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < npix;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    float vin[64];
    for (int c = 0; c < C; ++c) vin[c] = __bfloat162float(v[p * C + c]);
    float acc = b2[0];
    for (int j = 0; j < P; ++j) {
      float h = sb1[j];
      const float* q = sQ1 + j * C;
      for (int c = 0; c < C; ++c) h += q[c] * vin[c];
      acc += sQ2[j] * gelu(h);
    }
    out[p] = acc;
  }
}

// Backward of the projection given dout: dv (f32) and dQ1, db1, dQ2, db2.
// Tiles of 64 pixels; C = 64, P = 128; block 256.  Partials in registers.
__global__ void __launch_bounds__(256) fno_proj_bwd(const __nv_bfloat16* __restrict__ v,
                                                     const float* __restrict__ Q1, const float* __restrict__ b1,
                                                     const float* __restrict__ Q2, size_t npix,
                                                     const float* __restrict__ dout, float* __restrict__ dv,
                                                     float* __restrict__ dQ1, float* __restrict__ db1,
                                                     float* __restrict__ dQ2, float* __restrict__ db2) {
  constexpr int C = 64, P = 128, PT = 64;
  extern __shared__ float sm[];
  float* sQ1 = sm;              // [P][C]
  float* sv = sQ1 + P * C;      // [PT][C]
  float* sdh = sv + PT * C;     // [PT][P]
  float* sgh = sdh + PT * P;    // [PT][P]  dout * gelu(h)
  float* sd = sgh + PT * P;     // [PT]
  for (int t = threadIdx.x; t < P * C; t += blockDim.x) sQ1[t] = Q1[t];
  float gq1[32], gbias1 = 0.f, gq2 = 0.f, gb2 = 0.f;
#pragma unroll
  for (int q = 0; q < 32; ++q) gq1[q] = 0.f;
  const size_t tiles = (npix + PT - 1) / PT;
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t p0 = tile * PT;
    const int np = static_cast<int>(min(static_cast<size_t>(PT), npix - p0));
    __syncthreads();
    for (int t = threadIdx.x; t < PT * C; t += blockDim.x) {
      const int pl = t / C;
      sv[t] = pl < np ? __bfloat162float(v[(p0 + pl) * C + (t - pl * C)]) : 0.f;
    }
    for (int t = threadIdx.x; t < PT; t += blockDim.x) sd[t] = t < np ? dout[p0 + t] : 0.f;
    __syncthreads();
    for (int t = threadIdx.x; t < PT * P; t += blockDim.x) {
      const int pl = t / P, j = t - pl * P;
      float h = b1[j];
      const float* q = sQ1 + j * C;
      const float* vv = sv + pl * C;
#pragma unroll 8
      for (int c = 0; c < C; ++c) h += q[c] * vv[c];
      const float d = sd[pl];
      sdh[t] = d * Q2[j] * gelu_grad(h);
      sgh[t] = d * gelu(h);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < PT * C; t += blockDim.x) {
      const int pl = t / C, c = t - pl * C;
      if (pl >= np) continue;
      float acc = 0.f;
#pragma unroll 8
      for (int j = 0; j < P; ++j) acc += sQ1[j * C + c] * sdh[pl * P + j];
      dv[(p0 + pl) * C + c] = acc;
    }
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      const int pr = threadIdx.x + q * 256;  // (j, c)
      const int j = pr / C, c = pr - j * C;
      float acc = 0.f;
      for (int pl = 0; pl < PT; ++pl) acc += sdh[pl * P + j] * sv[pl * C + c];
      gq1[q] += acc;
    }
    if (threadIdx.x < P)
      for (int pl = 0; pl < PT; ++pl) {
        gbias1 += sdh[pl * P + threadIdx.x];
        gq2 += sgh[pl * P + threadIdx.x];
      }
    if (threadIdx.x == 0)
      for (int pl = 0; pl < PT; ++pl) gb2 += sd[pl];
  }
#pragma unroll
  for (int q = 0; q < 32; ++q) atomicAdd(dQ1 + threadIdx.x + q * 256, gq1[q]);
  if (threadIdx.x < P) {
    atomicAdd(db1 + threadIdx.x, gbias1);
    atomicAdd(dQ2 + threadIdx.x, gq2);
  }
  if (threadIdx.x == 0) atomicAdd(db2, gb2);
}

// Lift backward: dWl, dbl and the input gradient da = sum_c Wl[c][0] dv0[c].
// Thread (c, lane group) accumulates over pixels in registers; block 256, C = 64.
__global__ void __launch_bounds__(256) fno_lift_bwd(const float* __restrict__ a, const float* __restrict__ dv0,
                                                     int S, const float* __restrict__ Wl, size_t npix,
                                                     float* __restrict__ dWl, float* __restrict__ dbl,
                                                     float* __restrict__ da) {
  constexpr int C = 64;
  __shared__ float red[4][C][4];
  const int c = threadIdx.x % C, grp = threadIdx.x / C;  // 4 groups of 64
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  const size_t SS = static_cast<size_t>(S) * S;
  for (size_t p = blockIdx.x * 4 + grp; p < npix; p += static_cast<size_t>(gridDim.x) * 4) {
    const int pp = static_cast<int>(p % SS);
    const float gx = static_cast<float>(pp % S) / S, gy = static_cast<float>(pp / S) / S;
    const float d = dv0[p * C + c];
    s0 += d * a[p];
    s1 += d * gx;
    s2 += d * gy;
    s3 += d;
  }
  red[grp][c][0] = s0;
  red[grp][c][1] = s1;
  red[grp][c][2] = s2;
  red[grp][c][3] = s3;
  __syncthreads();
  if (threadIdx.x < C) {
    float t0 = 0.f, t1 = 0.f, t2 = 0.f, t3 = 0.f;
    for (int g = 0; g < 4; ++g) {
      t0 += red[g][threadIdx.x][0];
      t1 += red[g][threadIdx.x][1];
      t2 += red[g][threadIdx.x][2];
      t3 += red[g][threadIdx.x][3];
    }
    atomicAdd(dWl + threadIdx.x * 3, t0);
    atomicAdd(dWl + threadIdx.x * 3 + 1, t1);
    atomicAdd(dWl + threadIdx.x * 3 + 2, t2);
    atomicAdd(dbl + threadIdx.x, t3);
  }
  if (da)
    for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < npix;
         p += static_cast<size_t>(gridDim.x) * blockDim.x) {
      float acc = 0.f;
      for (int k = 0; k < C; ++k) acc += Wl[k * 3] * dv0[p * C + k];
      da[p] = acc;
    }
}

// MSE loss on [B][S][S]: dout = 2 (out - tgt) / n (and loss parts).
__global__ void fno_mse(const float* __restrict__ out, const float* __restrict__ tgt, size_t n,
                        float* __restrict__ dout, float* __restrict__ loss) {
  __shared__ float red[32];
  float s = 0.f;
  const float inv = 1.f / static_cast<float>(n);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float r = out[i] - tgt[i];
    if (dout) dout[i] = 2.f * r * inv;
    s += r * r * inv;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(loss, t);
  }
}

// Adam step on the flat parameter vector.
__global__ void fno_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                         float* __restrict__ m2, size_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                         float wd) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i] + wd * p[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
  }
}

}  // namespace huv_dev

// ================================================================== host
namespace huv {

struct Fno {
  int S, C, m, L, P, J, modes, B_cap = 0, device;
  size_t npar = 0;
  // parameter offsets (floats)
  size_t oWl, obl, oQ1, ob1, oQ2, ob2;
  std::vector<size_t> oR, oW, ob;
  float *par = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  float2 *twx = nullptr, *twy = nullptr;
  int64_t adam_t = 0;
  // activations
  std::vector<__nv_bfloat16*> v, z;
  std::vector<float2*> Xl;
  float2 *Xa = nullptr, *Y = nullptr, *Za = nullptr, *dX = nullptr;
  float *out = nullptr, *dout = nullptr, *dvA = nullptr, *dvB = nullptr, *dz = nullptr, *loss = nullptr;
  size_t act_bytes = 0;

  Fno(int S_, int C_, int m_, int L_, int P_, uint64_t seed, int dev) : S(S_), C(C_), m(m_), L(L_), P(P_), device(dev) {
    J = 2 * m;
    modes = J * m;
    size_t o = 0;
    oWl = o; o += C * 3;
    obl = o; o += C;
    for (int l = 0; l < L; ++l) {
      oR.push_back(o); o += static_cast<size_t>(modes) * C * C * 2;
      oW.push_back(o); o += static_cast<size_t>(C) * C;
      ob.push_back(o); o += C;
    }
    oQ1 = o; o += static_cast<size_t>(P) * C;
    ob1 = o; o += P;
    oQ2 = o; o += P;
    ob2 = o; o += 1;
    npar = o;
    std::vector<float> h(npar, 0.f);
    std::mt19937_64 rng(seed);
    auto uni = [&](float a, float b) { return std::uniform_real_distribution<float>(a, b)(rng); };
    const float sl = 1.f / std::sqrt(3.f), sc = 1.f / std::sqrt(static_cast<float>(C)),
                sp = 1.f / std::sqrt(static_cast<float>(P));
    for (int i = 0; i < C * 3; ++i) h[oWl + i] = uni(-sl, sl);
    for (int i = 0; i < C; ++i) h[obl + i] = uni(-sl, sl);
    const float sr = 1.f / (static_cast<float>(C) * C);
    for (int l = 0; l < L; ++l) {
      for (size_t i = 0; i < static_cast<size_t>(modes) * C * C * 2; ++i) h[oR[l] + i] = sr * uni(0.f, 1.f);
      for (int i = 0; i < C * C; ++i) h[oW[l] + i] = uni(-sc, sc);
      for (int i = 0; i < C; ++i) h[ob[l] + i] = uni(-sc, sc);
    }
    for (int i = 0; i < P * C; ++i) h[oQ1 + i] = uni(-sc, sc);
    for (int i = 0; i < P; ++i) h[ob1 + i] = uni(-sc, sc);
    for (int i = 0; i < P; ++i) h[oQ2 + i] = uni(-sp, sp);
    h[ob2] = 0.f;
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaMalloc(&par, npar * 4), "cudaMalloc(fno params)");
    check_cuda(cudaMalloc(&grad, npar * 4), "cudaMalloc(fno grad)");
    check_cuda(cudaMalloc(&m1, npar * 4), "cudaMalloc(fno m1)");
    check_cuda(cudaMalloc(&m2, npar * 4), "cudaMalloc(fno m2)");
    check_cuda(cudaMemcpy(par, h.data(), npar * 4, cudaMemcpyHostToDevice), "upload fno params");
    check_cuda(cudaMemset(m1, 0, npar * 4), "memset");
    check_cuda(cudaMemset(m2, 0, npar * 4), "memset");
    std::vector<float2> tx(static_cast<size_t>(m) * S), ty(static_cast<size_t>(J) * S);
    for (int k = 0; k < m; ++k)
      for (int x = 0; x < S; ++x) {
        const double a = -2.0 * 3.14159265358979323846 * k * static_cast<double>(x) / S;
        tx[static_cast<size_t>(k) * S + x] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
      }
    for (int j = 0; j < J; ++j) {
      const int ky = j < m ? j : j - J;
      for (int y = 0; y < S; ++y) {
        const double a = -2.0 * 3.14159265358979323846 * ky * static_cast<double>(y) / S;
        ty[static_cast<size_t>(j) * S + y] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
      }
    }
    check_cuda(cudaMalloc(&twx, tx.size() * 8), "cudaMalloc(twx)");
    check_cuda(cudaMalloc(&twy, ty.size() * 8), "cudaMalloc(twy)");
    check_cuda(cudaMemcpy(twx, tx.data(), tx.size() * 8, cudaMemcpyHostToDevice), "upload twx");
    check_cuda(cudaMemcpy(twy, ty.data(), ty.size() * 8, cudaMemcpyHostToDevice), "upload twy");
    static bool attr = false;
    if (!attr) {
      const int big = 200 * 1024;
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_dft_x<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_dft_x<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_proj, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_proj_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_layer_out, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      attr = true;
    }
  }

  void free_acts() {
    for (auto p : v) cudaFree(p);
    for (auto p : z) cudaFree(p);
    for (auto p : Xl) cudaFree(p);
    v.clear();
    z.clear();
    Xl.clear();
    cudaFree(Xa);
    cudaFree(Y);
    cudaFree(Za);
    cudaFree(dX);
    cudaFree(out);
    cudaFree(dout);
    cudaFree(dvA);
    cudaFree(dvB);
    cudaFree(dz);
    cudaFree(loss);
    Xa = Y = Za = dX = nullptr;
    out = dout = dvA = dvB = dz = loss = nullptr;
  }

  ~Fno() {
    cudaSetDevice(device);
    free_acts();
    cudaFree(par);
    cudaFree(grad);
    cudaFree(m1);
    cudaFree(m2);
    cudaFree(twx);
    cudaFree(twy);
  }

  void ensure(int B) {
    if (B <= B_cap) return;
    free_acts();
    const size_t pix = static_cast<size_t>(B) * S * S;
    auto al = [](void** p, size_t b) { check_cuda(cudaMalloc(p, b), "cudaMalloc(fno activations)"); };
    for (int l = 0; l <= L; ++l) {
      __nv_bfloat16* p;
      al(reinterpret_cast<void**>(&p), pix * C * 2);
      v.push_back(p);
    }
    for (int l = 0; l < L; ++l) {
      __nv_bfloat16* p;
      al(reinterpret_cast<void**>(&p), pix * C * 2);
      z.push_back(p);
      float2* x;
      al(reinterpret_cast<void**>(&x), static_cast<size_t>(B) * modes * C * 8);
      Xl.push_back(x);
    }
    al(reinterpret_cast<void**>(&Xa), static_cast<size_t>(B) * S * m * C * 8);
    al(reinterpret_cast<void**>(&Za), static_cast<size_t>(B) * S * m * C * 8);
    al(reinterpret_cast<void**>(&Y), static_cast<size_t>(B) * modes * C * 8);
    al(reinterpret_cast<void**>(&dX), static_cast<size_t>(B) * modes * C * 8);
    al(reinterpret_cast<void**>(&out), pix * 4);
    al(reinterpret_cast<void**>(&dout), pix * 4);
    al(reinterpret_cast<void**>(&dvA), pix * C * 4);
    al(reinterpret_cast<void**>(&dvB), pix * C * 4);
    al(reinterpret_cast<void**>(&dz), pix * C * 4);
    al(reinterpret_cast<void**>(&loss), 4);
    B_cap = B;
  }

  // images[b][S][S] = FNO(masks[b]); activations kept for backward.
  void forward(int B, const float* masks, float* images, cudaStream_t st) {
    using namespace huv_dev;
    ensure(B);
    const size_t pix = static_cast<size_t>(B) * S * S;
    fno_lift<<<2048, 256, 0, st>>>(masks, S, C, par + oWl, par + obl, v[0], pix * C);
    for (int l = 0; l < L; ++l) {
      fno_dft_x<__nv_bfloat16><<<dim3(S, B), 256, static_cast<size_t>(S) * C * 4, st>>>(v[l], S, C, m, twx, Xa);
      fno_dft_y<false><<<dim3(J, B), 256, 0, st>>>(Xa, S, C, m, twy, Xl[l]);
      fno_mix<<<dim3(modes, B), C, C * 8, st>>>(Xl[l], reinterpret_cast<const float2*>(par + oR[l]), C, modes, Y);
      fno_dft_y<true><<<dim3(S, B), 256, 0, st>>>(Y, S, C, m, twy, Za);
      fno_layer_out<<<dim3(S, B), 256, static_cast<size_t>(C) * C * 4 + static_cast<size_t>(m) * C * 8, st>>>(
          Za, v[l], par + oW[l], par + ob[l], S, C, m, twx, l < L - 1 ? 1 : 0, z[l], v[l + 1]);
    }
    fno_proj<<<1184, 256, (static_cast<size_t>(P) * C + 2 * P) * 4, st>>>(v[L], par + oQ1, par + ob1, par + oQ2,
                                                                         par + ob2, C, P, pix, images ? images : out);
    check_cuda(cudaGetLastError(), "fno forward");
  }

  // Backward from dout (device, [B][S][S]); accumulates into grad (zeroed
  // here) and writes the input gradient dmask when given.
  void backward(int B, const float* masks, const float* dOut, float* dmask, cudaStream_t st) {
    using namespace huv_dev;
    const size_t pix = static_cast<size_t>(B) * S * S;
    check_cuda(cudaMemsetAsync(grad, 0, npar * 4, st), "memset grad");
    const size_t smp = (static_cast<size_t>(P) * C + static_cast<size_t>(64) * C + 2 * static_cast<size_t>(64) * P + 64) * 4;
    fno_proj_bwd<<<1184, 256, smp, st>>>(v[L], par + oQ1, par + ob1, par + oQ2, pix, dOut, dvA, grad + oQ1,
                                         grad + ob1, grad + oQ2, grad + ob2);
    float* dnext = dvA;
    float* dcur = dvB;
    for (int l = L - 1; l >= 0; --l) {
      fno_layer_bwd<<<dim3(S, B), 256, 0, st>>>(dnext, z[l], v[l], par + oW[l], S, l < L - 1 ? 1 : 0, dz, dcur,
                                                 grad + oW[l], grad + ob[l]);
      fno_dft_x<float><<<dim3(S, B), 256, static_cast<size_t>(S) * C * 4, st>>>(dz, S, C, m, twx, Xa);
      fno_dft_y<false><<<dim3(J, B), 256, 0, st>>>(Xa, S, C, m, twy, Y);
      fno_scale_modes<<<256, 256, 0, st>>>(Y, B, J, m, C, 1.f / (static_cast<float>(S) * S));
      fno_mix_bwd<<<modes, 256, static_cast<size_t>(2) * B * C * 8, st>>>(
          Xl[l], Y, reinterpret_cast<const float2*>(par + oR[l]), C, modes, B, dX,
          reinterpret_cast<float2*>(grad + oR[l]));
      fno_dft_y<true><<<dim3(S, B), 256, 0, st>>>(dX, S, C, m, twy, Za);
      fno_spec_to_dv<<<dim3(S, B), 256, static_cast<size_t>(m) * C * 8, st>>>(Za, S, C, m, twx, dcur);
      std::swap(dnext, dcur);
    }
    fno_lift_bwd<<<1184, 256, 0, st>>>(masks, dnext, S, par + oWl, pix, grad + oWl, grad + obl, dmask);
    check_cuda(cudaGetLastError(), "fno backward");
  }

  float mse(int B, const float* targets, cudaStream_t st) {
    using namespace huv_dev;
    const size_t pix = static_cast<size_t>(B) * S * S;
    check_cuda(cudaMemsetAsync(loss, 0, 4, st), "memset loss");
    fno_mse<<<1184, 256, 0, st>>>(out, targets, pix, dout, loss);
    float h = 0;
    check_cuda(cudaMemcpyAsync(&h, loss, 4, cudaMemcpyDeviceToHost, st), "D2H loss");
    check_cuda(cudaStreamSynchronize(st), "sync");
    return h;
  }

  void adam(float lr, float wd, cudaStream_t st) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(adam_t)), c2 = 1.f - std::pow(b2, static_cast<float>(adam_t));
    huv_dev::fno_adam<<<1184, 256, 0, st>>>(par, grad, m1, m2, npar, lr, b1, b2, 1e-8f, c1, c2, wd);
    check_cuda(cudaGetLastError(), "fno adam");
  }
};

}  // namespace huv

namespace huv {
// The FNO as the image model of surrogate-assisted ILT.  input_grad reuses
// the activations of the preceding forward on the same maps.
struct FnoImageModel : Surrogate {
  Fno* f;
  explicit FnoImageModel(Fno* f_) : f(f_) {}
  int grid() const override { return f->S; }
  void forward(int B, const float* t, float* img, cudaStream_t st) override { f->forward(B, t, img, st); }
  void input_grad(int B, const float* t, const float* dout, float* dt, cudaStream_t st) override {
    f->backward(B, t, dout, dt, st);
  }
};
}  // namespace huv

using huv::Error;
using huv::Fno;

namespace {
template <typename F>
huv_status fno_guard(F&& f) {
  try {
    f();
    huv::set_last_error("");
    return HUV_OK;
  } catch (const Error& e) {
    huv::set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    huv::set_last_error(e.what());
    return HUV_ERR_NUMERICAL;
  }
}
Fno* as_fno(void* p) {
  if (!p) throw Error(HUV_ERR_INVALID_PARAMETER, "fno: null handle");
  return static_cast<Fno*>(p);
}
}  // namespace

extern "C" {

huv_status huv_fno_create(int32_t grid, int32_t width, int32_t modes, int32_t layers, int32_t proj, uint64_t seed,
                          int32_t device, void** fno_out) {
  return fno_guard([&] {
    if (!fno_out) throw Error(HUV_ERR_INVALID_PARAMETER, "fno_out: null");
    if (width != 64 || proj != 128)
      throw Error(HUV_ERR_UNSUPPORTED, "fno: this build's kernels are specialised to width 64, projection 128");
    if (grid < 8 || (grid & (grid - 1)) || modes < 1 || 2 * modes > grid || layers < 1)
      throw Error(HUV_ERR_INVALID_PARAMETER, "fno: grid power of two >= 8, 1 <= modes <= grid/2, layers >= 1");
    *fno_out = new Fno(grid, width, modes, layers, proj, seed, device);
  });
}

void huv_fno_destroy(void* fno) { delete static_cast<Fno*>(fno); }

huv_status huv_fno_params(void* fno, float* host, int64_t capacity, int64_t* count) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    if (count) *count = static_cast<int64_t>(f->npar);
    if (!host) return;
    if (capacity < static_cast<int64_t>(f->npar)) throw Error(HUV_ERR_DIMENSION_MISMATCH, "fno params: capacity");
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    huv::check_cuda(cudaMemcpy(host, f->par, f->npar * 4, cudaMemcpyDeviceToHost), "D2H params");
  });
}

huv_status huv_fno_set_params(void* fno, const float* host, int64_t count) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    if (!host || count != static_cast<int64_t>(f->npar)) throw Error(HUV_ERR_DIMENSION_MISMATCH, "fno params: count");
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    huv::check_cuda(cudaMemcpy(f->par, host, f->npar * 4, cudaMemcpyHostToDevice), "H2D params");
  });
}

huv_status huv_fno_forward(void* fno, int32_t batch, const float* masks, float* images, void* stream) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    if (batch <= 0 || !masks || !images) throw Error(HUV_ERR_INVALID_PARAMETER, "fno forward: arguments");
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    f->forward(batch, masks, images, static_cast<cudaStream_t>(stream));
  });
}

// Gradients: with targets, of the MSE loss (loss_host receives it); without,
// of sum(dout . FNO(masks)).  param_grad (device, npar floats) and dmask
// (device, batch*S*S) are optional outputs.
huv_status huv_fno_backward(void* fno, int32_t batch, const float* masks, const float* targets, const float* dout,
                            float* param_grad, float* dmask, float* loss_host, void* stream) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    if (batch <= 0 || !masks || (!targets && !dout)) throw Error(HUV_ERR_INVALID_PARAMETER, "fno backward: arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    f->forward(batch, masks, nullptr, st);
    const float* d = dout;
    if (targets) {
      const float l = f->mse(batch, targets, st);
      if (loss_host) *loss_host = l;
      d = f->dout;
    }
    f->backward(batch, masks, d, dmask, st);
    if (param_grad)
      huv::check_cuda(cudaMemcpyAsync(param_grad, f->grad, f->npar * 4, cudaMemcpyDeviceToDevice, st), "copy grad");
  });
}

huv_status huv_fno_train_step(void* fno, int32_t batch, const float* masks, const float* targets, float lr,
                              float weight_decay, float* loss_host, void* stream) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    if (batch <= 0 || !masks || !targets || !(lr > 0)) throw Error(HUV_ERR_INVALID_PARAMETER, "fno train: arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    f->forward(batch, masks, nullptr, st);
    const float l = f->mse(batch, targets, st);
    if (loss_host) *loss_host = l;
    f->backward(batch, masks, f->dout, nullptr, st);
    f->adam(lr, weight_decay, st);
  });
}

huv_status huv_ilt_optimize_surrogate(void* engine, void* fno, const huv_ilt_params* params, const huv_ilt_opt* opt,
                                      int32_t n_masks, float* theta, const float* target, huv_surrogate_ilt* sur,
                                      double* final_cost, int32_t* iterations, double* history, void* stream) {
  return fno_guard([&] {
    huv::Engine* e = static_cast<huv::Engine*>(engine);
    Fno* f = as_fno(fno);
    if (!e || !params || !opt || !theta || !target || !sur)
      throw Error(HUV_ERR_INVALID_PARAMETER, "surrogate ilt: null argument");
    if (opt->max_iterations < 0 || !(opt->learning_rate > 0) || !(opt->convergence_tol >= 0))
      throw Error(HUV_ERR_INVALID_PARAMETER, "ilt optimizer: max_iterations >= 0, learning_rate > 0, tol >= 0");
    if (sur->judge_every < 1 || !(sur->error_bound > 0))
      throw Error(HUV_ERR_INVALID_PARAMETER, "surrogate ilt: judge_every >= 1, error_bound > 0");
    if (f->S != e->n) throw Error(HUV_ERR_DIMENSION_MISMATCH, "surrogate ilt: FNO grid differs from the engine grid");
    if (!(params->beta > 0) || !(params->absorber >= 0 && params->absorber < 1) || !(params->tv_epsilon > 0) ||
        (params->cost_kind != 0 && params->cost_kind != 1))
      throw Error(HUV_ERR_INVALID_PARAMETER, "ilt: invalid params");
    if (n_masks <= 0) return;
    std::lock_guard<std::mutex> lock(e->mu);
    e->ensure_device();
    huv::FnoImageModel model(f);
    huv::SurrogateReport rep;
    e->ilt_optimize(*params, *opt, n_masks, theta, target, final_cost, iterations, history,
                    static_cast<cudaStream_t>(stream), &model, sur->judge_every, sur->error_bound, &rep);
    sur->surrogate_iterations = rep.surrogate_iterations;
    sur->exact_iterations = rep.exact_iterations;
    sur->takeover_iteration = rep.takeover_iteration;
    sur->n_judges = static_cast<int32_t>(rep.judge_errors.size());
    for (int i = 0; i < 64; ++i)
      sur->judge_errors[i] = i < static_cast<int>(rep.judge_errors.size()) ? rep.judge_errors[i] : 0.0;
  });
}

}  // extern "C"
