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

namespace huv_launch {
// tensor-core forward of the FNO (csrc/cuda/fno_tc.cu)
cudaError_t fno_tc_set_smem();
bool fno_tc_proj_bwd(size_t pix, const __nv_bfloat16* v, const float* Q1, const float* b1, const float* q2,
                     const float* dout, float* dv, float* dQ1, float* db1, float* dQ2, float* db2, int* err,
                     cudaStream_t st);
bool fno_tc_layer_bwd(size_t pix, const float* dvnext, const __nv_bfloat16* z, const __nv_bfloat16* v, const float* W,
                      int act, float* dz, float* dv, float* dW, float* db, int* err, cudaStream_t st);
bool fno_tc_layer(int B, int S, int m, const __nv_bfloat16* v, const __nv_bfloat16* Wb, const __nv_bfloat16* Tw,
                  const __nv_bfloat16* Zs, const float* bias, int act, __nv_bfloat16* zsave, __nv_bfloat16* vnext,
                  int* err, cudaStream_t st);
bool fno_tc_proj(int B, int S, const __nv_bfloat16* v, const __nv_bfloat16* Q1b, const float* b1, const float* q2,
                 const float* b2, float* out, int* err, cudaStream_t st);
void fno_tc_to_bf16(const float* a, int n, __nv_bfloat16* b, cudaStream_t st);
void fno_tc_pack_zs(const float2* Z, int rows, int m, int S, __nv_bfloat16* Zs, cudaStream_t st);
void fno_tc_tw_table(const float2* twx, int S, int m, __nv_bfloat16* Tw, cudaStream_t st);
}  // namespace huv_launch

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

// ------------------------------------------------------------ register tiles
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
// acc[p][q] += a[p] w[q]
__device__ __forceinline__ void fma44(float (&acc)[4][4], float4 a, float4 w) {
  const float av[4] = {a.x, a.y, a.z, a.w}, wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(av[p], wv[q], acc[p][q]);
}
__device__ __forceinline__ void st_bf16x4(__nv_bfloat16* p, float a, float b, float c, float d) {
  __nv_bfloat162 lo = __floats2bfloat162_rn(a, b), hi = __floats2bfloat162_rn(c, d);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t*>(&lo);
  u.y = *reinterpret_cast<uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(p) = u;
}

// ------------------------------------------------------------ DFT along x
// out[r][kx][c] (complex) = sum_x in[r][x][c] e^{-2 pi i kx x / S} for rows r
// (= (b, y)), kx < m <= 16, C = 64.  Rows are grid-strided; x runs in chunks
// of up to 128 split over four thread groups; thread (kg, cg) of a group owns
// kx 4kg..4kg+3 x c 4cg..4cg+3 (complex), the groups are summed at the end.
// Dynamic shared memory: 48 KiB.
template <typename T>
__global__ void __launch_bounds__(256) fno_dft_x(const T* __restrict__ in, int S, int m,
                                                  const float2* __restrict__ twx, float2* __restrict__ out,
                                                  int rows) {
  constexpr int C = 64, XC = 128;
  extern __shared__ __align__(16) float dsm[];
  float* sIn = dsm;                                        // [XC][C]
  float2* sTw = reinterpret_cast<float2*>(sIn + XC * C);   // [16][XC]
  float2* red = reinterpret_cast<float2*>(sIn);            // [4][16][C], aliases sIn
  const int t = threadIdx.x;
  const int grp = t >> 6, kg = t & 3, cg = (t >> 2) & 15;
  const int xc = min(XC, S), xs = xc >> 2;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    float acc[4][4][2];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[q][c][0] = acc[q][c][1] = 0.f;
    const size_t row = static_cast<size_t>(r) * S * C;
    for (int x0 = 0; x0 < S; x0 += xc) {
      __syncthreads();
      for (int e = t; e < xc * C; e += 256) sIn[e] = ld(in, row + static_cast<size_t>(x0) * C + e);
      for (int e = t; e < 16 * xc; e += 256) {
        const int kx = e / xc, x = e - kx * xc;
        sTw[e] = kx < m ? __ldg(twx + static_cast<size_t>(kx) * S + x0 + x) : make_float2(0.f, 0.f);
      }
      __syncthreads();
      for (int xx = 0; xx < xs; ++xx) {
        const int x = grp * xs + xx;
        const float4 a = ld4(sIn + x * C + cg * 4);
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 w = sTw[(kg * 4 + q) * xc + x];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            acc[q][c][0] = fmaf(av[c], w.x, acc[q][c][0]);
            acc[q][c][1] = fmaf(av[c], w.y, acc[q][c][1]);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 4; ++c)
        red[(grp * 16 + kg * 4 + q) * C + cg * 4 + c] = make_float2(acc[q][c][0], acc[q][c][1]);
    __syncthreads();
    for (int e = t; e < m * C; e += 256) {
      float2 sum = red[e];
#pragma unroll
      for (int g = 1; g < 4; ++g) {
        const float2 v = red[g * 16 * C + e];
        sum.x += v.x;
        sum.y += v.y;
      }
      out[static_cast<size_t>(r) * m * C + e] = sum;
    }
  }
}

// ------------------------------------------------------------ DFT along y
// Forward (to modes): out[b][j][col] = sum_y in[b][y][col] twy[j][y], col =
// (kx, c) over m * C columns; grid (ceil(mC / 64), B), thread (col, j group
// of 8), J = 2m <= 32.
// Inverse (from modes): out[b][y][col] = sum_j in[b][j][col] conj(twy[j][y]);
// grid (S, B).  twy[j][y] = e^{-2 pi i ky_j y / S}.
template <bool INVERSE>
__global__ void __launch_bounds__(256) fno_dft_y(const float2* __restrict__ in, int S, int C, int m,
                                                  const float2* __restrict__ twy, float2* __restrict__ out) {
  const int J = 2 * m, mC = m * C;
  if (!INVERSE) {
    const int b = blockIdx.y;
    const int col = blockIdx.x * 64 + (threadIdx.x & 63);
    const int j0 = (threadIdx.x >> 6) * 8;
    if (col >= mC || j0 >= J) return;
    float2 acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = make_float2(0.f, 0.f);
    const float2* src = in + static_cast<size_t>(b) * S * mC + col;
    for (int y = 0; y < S; ++y) {
      const float2 v = src[static_cast<size_t>(y) * mC];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (j0 + q < J) {
          const float2 w = __ldg(twy + static_cast<size_t>(j0 + q) * S + y);
          acc[q].x = fmaf(v.x, w.x, fmaf(-v.y, w.y, acc[q].x));
          acc[q].y = fmaf(v.x, w.y, fmaf(v.y, w.x, acc[q].y));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (j0 + q < J) out[(static_cast<size_t>(b) * J + j0 + q) * mC + col] = acc[q];
  } else {
    const int r = blockIdx.x, b = blockIdx.y;
    for (int t = threadIdx.x; t < mC; t += blockDim.x) {
      float re = 0.f, im = 0.f;
      for (int q = 0; q < J; ++q) {
        const float2 v = in[(static_cast<size_t>(b) * J + q) * mC + t];
        float2 w = __ldg(twy + static_cast<size_t>(q) * S + r);
        w.y = -w.y;
        re += v.x * w.x - v.y * w.y;
        im += v.x * w.y + v.y * w.x;
      }
      out[(static_cast<size_t>(b) * S + r) * mC + t] = make_float2(re, im);
    }
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
// z = S^-2 Re sum_kx w_kx Z[r][kx][o] e^{+i th} + sum_i W[o][i] v[i] + b[o],
// th = 2 pi kx x / S; v_next = GELU(z) (or z for the last layer).  Rows r =
// (b, y) grid-strided; pixels in tiles of 64; thread (pg, og) owns pixels
// 4pg..4pg+3 x outputs 4og..4og+3.  The spectral term is a K = 2m
// contraction of cos/sin rows against (w Re Z, -w Im Z).
// Dynamic shared memory: (2 * 64 * 68 + 2m * (64 + 68)) floats.
__global__ void __launch_bounds__(256) fno_layer_out(const float2* __restrict__ Z, const __nv_bfloat16* __restrict__ v,
                                                      const float* __restrict__ W, const float* __restrict__ bias,
                                                      int S, int m, const float2* __restrict__ twx, int act,
                                                      __nv_bfloat16* __restrict__ zsave,
                                                      __nv_bfloat16* __restrict__ vnext, int rows) {
  constexpr int C = 64, XT = 64, LD = 68;
  extern __shared__ __align__(16) float dsm[];
  float* sWT = dsm;             // [i][LD]: W transposed
  float* sV = sWT + C * LD;     // [i][LD]: v tile transposed
  float* sZ = sV + C * LD;      // [2m][C]
  float* sT = sZ + 2 * m * C;   // [2m][LD]
  const int t = threadIdx.x, og = t & 15, pg = t >> 4;
  for (int e = t; e < C * C; e += 256) sWT[(e & 63) * LD + (e >> 6)] = W[e];
  float b4[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) b4[q] = bias[og * 4 + q];
  const float inv = 1.f / (static_cast<float>(S) * S);
  const int xt = min(XT, S);
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    __syncthreads();
    const float2* Zr = Z + static_cast<size_t>(r) * m * C;
    for (int e = t; e < m * C; e += 256) {
      const int kx = e / C, o = e - kx * C;
      const float w = (kx == 0 ? 1.f : 2.f) * inv;
      const float2 zz = Zr[e];
      sZ[(2 * kx) * C + o] = w * zz.x;
      sZ[(2 * kx + 1) * C + o] = -w * zz.y;
    }
    const size_t row = static_cast<size_t>(r) * S * C;
    for (int x0 = 0; x0 < S; x0 += xt) {
      __syncthreads();
      for (int e = t; e < xt * C; e += 256)
        sV[(e & 63) * LD + (e >> 6)] = __bfloat162float(v[row + static_cast<size_t>(x0) * C + e]);
      for (int e = t; e < 2 * m * xt; e += 256) {
        const int kk = e / xt, px = e - kk * xt;
        const float2 w = __ldg(twx + static_cast<size_t>(kk >> 1) * S + x0 + px);  // (cos, -sin)
        sT[kk * LD + px] = (kk & 1) ? -w.y : w.x;
      }
      __syncthreads();
      if (pg * 4 < xt) {
        float acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = b4[q];
#pragma unroll 8
        for (int i = 0; i < C; ++i) fma44(acc, ld4(sV + i * LD + pg * 4), ld4(sWT + i * LD + og * 4));
        for (int kk = 0; kk < 2 * m; ++kk) fma44(acc, ld4(sT + kk * LD + pg * 4), ld4(sZ + kk * C + og * 4));
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const size_t g = row + static_cast<size_t>(x0 + pg * 4 + p) * C + og * 4;
          st_bf16x4(zsave + g, acc[p][0], acc[p][1], acc[p][2], acc[p][3]);
          if (act)
            st_bf16x4(vnext + g, gelu(acc[p][0]), gelu(acc[p][1]), gelu(acc[p][2]), gelu(acc[p][3]));
          else
            st_bf16x4(vnext + g, acc[p][0], acc[p][1], acc[p][2], acc[p][3]);
        }
      }
    }
  }
}

// Backward of the layer output: dz = dvnext * GELU'(z) (or dvnext) -> dz
// (f32); dv = W^T dz (f32, overwriting dv); dW += dz^T v; db += sum dz.  Rows
// grid-strided, tiles of 64 pixels; weight-gradient partials stay in
// registers (thread (og, ig) owns 4 x 4 of dW) until one atomic add per block.
// Dynamic shared memory: (64 * 64 + 3 * 64 * 68) floats.
__global__ void __launch_bounds__(256) fno_layer_bwd(const float* __restrict__ dvnext,
                                                      const __nv_bfloat16* __restrict__ z,
                                                      const __nv_bfloat16* __restrict__ v,
                                                      const float* __restrict__ W, int S, int act,
                                                      float* __restrict__ dz, float* __restrict__ dv,
                                                      float* __restrict__ dW, float* __restrict__ db, int rows) {
  constexpr int C = 64, XT = 64, LD = 68;
  extern __shared__ __align__(16) float dsm[];
  float* sW = dsm;             // [o][C]
  float* sD = sW + C * C;      // [px][LD]  dz
  float* sDT = sD + XT * LD;   // [o][LD]   dz transposed
  float* sV = sDT + C * LD;    // [px][LD]
  const int t = threadIdx.x, hi = t >> 4, lo = t & 15;
  for (int e = t; e < C * C; e += 256) sW[e] = W[e];
  float gw[4][4], gb = 0.f;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) gw[p][q] = 0.f;
  const int xt = min(XT, S);
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const size_t row = static_cast<size_t>(r) * S * C;
    for (int x0 = 0; x0 < S; x0 += xt) {
      __syncthreads();
      for (int e = t; e < xt * C; e += 256) {
        const int px = e >> 6, o = e & 63;
        const size_t g = row + static_cast<size_t>(x0) * C + e;
        const float gv = dvnext[g];
        const float d = act ? gv * gelu_grad(__bfloat162float(z[g])) : gv;
        dz[g] = d;
        sD[px * LD + o] = d;
        sDT[o * LD + px] = d;
        sV[px * LD + o] = __bfloat162float(v[g]);
      }
      __syncthreads();
      if (hi * 4 < xt) {
        float acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = 0.f;
#pragma unroll 8
        for (int o = 0; o < C; ++o) fma44(acc, ld4(sDT + o * LD + hi * 4), ld4(sW + o * C + lo * 4));
#pragma unroll
        for (int p = 0; p < 4; ++p)
          *reinterpret_cast<float4*>(dv + row + static_cast<size_t>(x0 + hi * 4 + p) * C + lo * 4) =
              make_float4(acc[p][0], acc[p][1], acc[p][2], acc[p][3]);
      }
#pragma unroll 4
      for (int px = 0; px < xt; ++px) fma44(gw, ld4(sD + px * LD + hi * 4), ld4(sV + px * LD + lo * 4));
      if (t < C)
        for (int px = 0; px < xt; ++px) gb += sD[px * LD + t];
    }
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) atomicAdd(dW + (hi * 4 + p) * C + lo * 4 + q, gw[p][q]);
  if (t < C) atomicAdd(db + t, gb);
}

// dv[r][x][c] += Re sum_kx Z[r][kx][c] e^{+2 pi i kx x / S} (weight 1); rows
// grid-strided, tiles of 64 pixels, thread (pg, cg) owns 4 x 4.
// Dynamic shared memory: 2m * (64 + 68) floats.
__global__ void __launch_bounds__(256) fno_spec_to_dv(const float2* __restrict__ Z, int S, int m,
                                                       const float2* __restrict__ twx, float* __restrict__ dv,
                                                       int rows) {
  constexpr int C = 64, XT = 64, LD = 68;
  extern __shared__ __align__(16) float dsm[];
  float* sZ = dsm;              // [2m][C]
  float* sT = sZ + 2 * m * C;   // [2m][LD]
  const int t = threadIdx.x, cg = t & 15, pg = t >> 4;
  const int xt = min(XT, S);
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    __syncthreads();
    const float2* Zr = Z + static_cast<size_t>(r) * m * C;
    for (int e = t; e < m * C; e += 256) {
      const int kx = e / C, c = e - kx * C;
      const float2 zz = Zr[e];
      sZ[(2 * kx) * C + c] = zz.x;
      sZ[(2 * kx + 1) * C + c] = -zz.y;
    }
    const size_t row = static_cast<size_t>(r) * S * C;
    for (int x0 = 0; x0 < S; x0 += xt) {
      __syncthreads();
      for (int e = t; e < 2 * m * xt; e += 256) {
        const int kk = e / xt, px = e - kk * xt;
        const float2 w = __ldg(twx + static_cast<size_t>(kk >> 1) * S + x0 + px);
        sT[kk * LD + px] = (kk & 1) ? -w.y : w.x;
      }
      __syncthreads();
      if (pg * 4 < xt) {
        float acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = 0.f;
        for (int kk = 0; kk < 2 * m; ++kk) fma44(acc, ld4(sT + kk * LD + pg * 4), ld4(sZ + kk * C + cg * 4));
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          float4* d = reinterpret_cast<float4*>(dv + row + static_cast<size_t>(x0 + pg * 4 + p) * C + cg * 4);
          float4 cur = *d;
          cur.x += acc[p][0];
          cur.y += acc[p][1];
          cur.z += acc[p][2];
          cur.w += acc[p][3];
          *d = cur;
        }
      }
    }
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
// out[p] = sum_j Q2[j] GELU(sum_c Q1[j][c] v[p][c] + b1[j]) + b2 (C = 64,
// P = 128).  Tiles of 64 pixels grid-strided; thread (pg, jg) owns pixels
// 4pg..4pg+3 x hidden units 8jg..8jg+7; the 16 j groups of a pixel quad sit
// in adjacent lanes and are summed with shuffles.
// Dynamic shared memory: (64 * 128 + 64 * 68) floats.
__global__ void __launch_bounds__(256) fno_proj(const __nv_bfloat16* __restrict__ v, const float* __restrict__ Q1,
                                                 const float* __restrict__ b1, const float* __restrict__ Q2,
                                                 const float* __restrict__ b2, size_t npix, float* __restrict__ out) {
  constexpr int C = 64, P = 128, PT = 64, LD = 68;
  extern __shared__ __align__(16) float dsm[];
  float* sQT = dsm;            // [c][P]
  float* sVT = sQT + C * P;    // [c][LD]
  const int t = threadIdx.x, jg = t & 15, pg = t >> 4;
  for (int e = t; e < C * P; e += 256) sQT[e] = Q1[(e & (P - 1)) * C + (e >> 7)];
  float bj[8], qj[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    bj[q] = b1[jg * 8 + q];
    qj[q] = Q2[jg * 8 + q];
  }
  const float bias2 = b2[0];
  const size_t tiles = (npix + PT - 1) / PT;
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t p0 = tile * PT;
    __syncthreads();
    for (int e = t; e < PT * C; e += 256) {
      const int px = e >> 6, c = e & 63;
      sVT[c * LD + px] = p0 + px < npix ? __bfloat162float(v[p0 * C + e]) : 0.f;
    }
    __syncthreads();
    float h[4][8];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 8; ++q) h[p][q] = bj[q];
#pragma unroll 4
    for (int c = 0; c < C; ++c) {
      const float4 a = ld4(sVT + c * LD + pg * 4);
      const float4 w0 = ld4(sQT + c * P + jg * 8), w1 = ld4(sQT + c * P + jg * 8 + 4);
      const float av[4] = {a.x, a.y, a.z, a.w};
      const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 8; ++q) h[p][q] = fmaf(av[p], wv[q], h[p][q]);
    }
    float part[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      float sum = 0.f;
#pragma unroll
      for (int q = 0; q < 8; ++q) sum = fmaf(qj[q], gelu(h[p][q]), sum);
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      part[p] = sum;
    }
    if (jg == 0)
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p0 + pg * 4 + p < npix) out[p0 + pg * 4 + p] = part[p] + bias2;
  }
}

// Backward of the projection given dout: dv (f32) and dQ1, db1, dQ2, db2.
// Per tile of 64 pixels: the hidden layer is recomputed (thread (pg, jg) as
// in the forward), dh = dout Q2 GELU'(h) is kept in shared memory in both
// orientations, dv = Q1^T dh (thread (pg, cg), 4 x 4) and dQ1 += dh^T v
// (thread (jg8, cg), 8 x 4 in registers across tiles).
// Dynamic shared memory: (2 * 64 * 128 + 2 * 64 * 68 + 64 * 132 + 128 * 68 + 64) floats.
__global__ void __launch_bounds__(256) fno_proj_bwd(const __nv_bfloat16* __restrict__ v,
                                                     const float* __restrict__ Q1, const float* __restrict__ b1,
                                                     const float* __restrict__ Q2, size_t npix,
                                                     const float* __restrict__ dout, float* __restrict__ dv,
                                                     float* __restrict__ dQ1, float* __restrict__ db1,
                                                     float* __restrict__ dQ2, float* __restrict__ db2) {
  constexpr int C = 64, P = 128, PT = 64, LD = 68, LDP = 132;
  extern __shared__ __align__(16) float dsm[];
  float* sQT = dsm;              // [c][P]
  float* sQ = sQT + C * P;       // [j][C]
  float* sVT = sQ + P * C;       // [c][LD]
  float* sV = sVT + C * LD;      // [px][LD]
  float* sDh = sV + PT * LD;     // [px][LDP]
  float* sDhT = sDh + PT * LDP;  // [j][LD]
  float* sd = sDhT + P * LD;     // [PT]
  const int t = threadIdx.x, hi = t >> 4, lo = t & 15;
  for (int e = t; e < C * P; e += 256) {
    sQT[e] = Q1[(e & (P - 1)) * C + (e >> 7)];
    sQ[e] = Q1[e];
  }
  float bj[8], qj[8], gb1[8], gq2[8], gq1[8][4], gd2 = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    bj[q] = b1[lo * 8 + q];
    qj[q] = Q2[lo * 8 + q];
    gb1[q] = gq2[q] = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) gq1[q][c] = 0.f;
  }
  const size_t tiles = (npix + PT - 1) / PT;
  for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const size_t p0 = tile * PT;
    __syncthreads();
    for (int e = t; e < PT * C; e += 256) {
      const int px = e >> 6, c = e & 63;
      const float x = p0 + px < npix ? __bfloat162float(v[p0 * C + e]) : 0.f;
      sVT[c * LD + px] = x;
      sV[px * LD + c] = x;
    }
    for (int e = t; e < PT; e += 256) sd[e] = p0 + e < npix ? dout[p0 + e] : 0.f;
    __syncthreads();
    {
      // hidden layer: thread (pg = hi, jg = lo)
      float h[4][8];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 8; ++q) h[p][q] = bj[q];
#pragma unroll 4
      for (int c = 0; c < C; ++c) {
        const float4 a = ld4(sVT + c * LD + hi * 4);
        const float4 w0 = ld4(sQT + c * P + lo * 8), w1 = ld4(sQT + c * P + lo * 8 + 4);
        const float av[4] = {a.x, a.y, a.z, a.w};
        const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 8; ++q) h[p][q] = fmaf(av[p], wv[q], h[p][q]);
      }
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int px = hi * 4 + p;
        const float d = sd[px];
        if (lo == 0) gd2 += d;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float hh = h[p][q];
          const float dh = d * qj[q] * gelu_grad(hh);
          gq2[q] = fmaf(d, gelu(hh), gq2[q]);
          gb1[q] += dh;
          sDh[px * LDP + lo * 8 + q] = dh;
          sDhT[(lo * 8 + q) * LD + px] = dh;
        }
      }
    }
    __syncthreads();
    {
      // dv: thread (pg = hi, cg = lo)
      float acc[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = 0.f;
#pragma unroll 8
      for (int j = 0; j < P; ++j) fma44(acc, ld4(sDhT + j * LD + hi * 4), ld4(sQ + j * C + lo * 4));
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p0 + hi * 4 + p < npix)
          *reinterpret_cast<float4*>(dv + (p0 + hi * 4 + p) * C + lo * 4) =
              make_float4(acc[p][0], acc[p][1], acc[p][2], acc[p][3]);
    }
    // dQ1: thread (jg8 = hi, cg = lo)
#pragma unroll 2
    for (int px = 0; px < PT; ++px) {
      const float4 a0 = ld4(sDh + px * LDP + hi * 8), a1 = ld4(sDh + px * LDP + hi * 8 + 4);
      const float4 b = ld4(sV + px * LD + lo * 4);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int c = 0; c < 4; ++c) gq1[q][c] = fmaf(av[q], bv[c], gq1[q][c]);
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int c = 0; c < 4; ++c) atomicAdd(dQ1 + (hi * 8 + q) * C + lo * 4 + c, gq1[q][c]);
  // gb1, gq2 (thread (pg = hi, jg = lo)): lanes l and l ^ 16 share jg.
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    gb1[q] += __shfl_xor_sync(0xffffffffu, gb1[q], 16);
    gq2[q] += __shfl_xor_sync(0xffffffffu, gq2[q], 16);
  }
  gd2 += __shfl_xor_sync(0xffffffffu, gd2, 16);
  if ((t & 31) < 16) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      atomicAdd(db1 + lo * 8 + q, gb1[q]);
      atomicAdd(dQ2 + lo * 8 + q, gq2[q]);
    }
    if (lo == 0) atomicAdd(db2, gd2);
  }
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
  // tensor-core forward (grids of at least 128): bf16 weights, twiddle table,
  // packed spectral operand, device error flag
  bool tc = false;
  __nv_bfloat16 *wb = nullptr, *q1b = nullptr, *tw_tab = nullptr, *zs = nullptr;
  int* tc_err = nullptr;
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
    static std::atomic<uint64_t> attr{0};
    huv::once_per_device(attr, [] {
      const int big = 200 * 1024;
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_dft_x<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_dft_x<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_proj, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_proj_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_layer_out, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
      check_cuda(cudaFuncSetAttribute(huv_dev::fno_spec_to_dv, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    });
    tc = S >= 128 && S % 128 == 0 && C == 64 && P == 128 && m <= 16;
    if (tc) {
      check_cuda(huv_launch::fno_tc_set_smem(), "cudaFuncSetAttribute(fno tc)");
      check_cuda(cudaMalloc(&wb, static_cast<size_t>(L) * C * C * 2), "cudaMalloc(fno wb)");
      check_cuda(cudaMalloc(&q1b, static_cast<size_t>(P) * C * 2), "cudaMalloc(fno q1b)");
      check_cuda(cudaMalloc(&tw_tab, static_cast<size_t>(S) * 64 * 2), "cudaMalloc(fno tw)");
      check_cuda(cudaMalloc(&tc_err, sizeof(int)), "cudaMalloc(fno err)");
      check_cuda(cudaMemset(tc_err, 0, sizeof(int)), "memset");
      huv_launch::fno_tc_tw_table(twx, S, m, tw_tab, nullptr);
      check_cuda(cudaDeviceSynchronize(), "fno_tw_table");
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
    cudaFree(zs);
    zs = nullptr;
    Xa = Y = Za = dX = nullptr;
    out = dout = dvA = dvB = dz = loss = nullptr;
  }

  ~Fno() {
    cudaSetDevice(device);
    free_acts();
    cudaFree(wb);
    cudaFree(q1b);
    cudaFree(tw_tab);
    cudaFree(tc_err);
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
    if (tc) al(reinterpret_cast<void**>(&zs), static_cast<size_t>(B) * S * 64 * 64 * 2);
    B_cap = B;
  }

  // Launch shapes and dynamic shared memory of the tiled kernels.
  static constexpr size_t kDftXSmem = (128 * 64 + 16 * 128 * 2) * 4;
  static constexpr size_t kProjSmem = (64 * 128 + 64 * 68) * 4;
  static constexpr size_t kProjBwdSmem = (2 * 64 * 128 + 2 * 64 * 68 + 64 * 132 + 128 * 68 + 64) * 4;
  static constexpr size_t kLayerBwdSmem = (64 * 64 + 3 * 64 * 68) * 4;
  size_t layer_out_smem() const { return (2 * 64 * 68 + 2 * static_cast<size_t>(m) * (64 + 68)) * 4; }
  size_t spec_smem() const { return (2 * static_cast<size_t>(m) * (64 + 68)) * 4; }
  static unsigned pgrid(size_t pix) { return static_cast<unsigned>(std::min<size_t>((pix + 63) / 64, 296)); }

  // images[b][S][S] = FNO(masks[b]); activations kept for backward.
  void forward(int B, const float* masks, float* images, cudaStream_t st) {
    using namespace huv_dev;
    ensure(B);
    const size_t pix = static_cast<size_t>(B) * S * S;
    const int rows = B * S;
    const dim3 rgrid(std::min(rows, 4096));
    const dim3 ygrid((m * C + 63) / 64, B);
    fno_lift<<<2048, 256, 0, st>>>(masks, S, C, par + oWl, par + obl, v[0], pix * C);
    for (int l = 0; l < L; ++l) {
      fno_dft_x<__nv_bfloat16><<<rgrid, 256, kDftXSmem, st>>>(v[l], S, m, twx, Xa, rows);
      fno_dft_y<false><<<ygrid, 256, 0, st>>>(Xa, S, C, m, twy, Xl[l]);
      fno_mix<<<dim3(modes, B), C, C * 8, st>>>(Xl[l], reinterpret_cast<const float2*>(par + oR[l]), C, modes, Y);
      fno_dft_y<true><<<dim3(S, B), 256, 0, st>>>(Y, S, C, m, twy, Za);
      if (tc) {
        huv_launch::fno_tc_to_bf16(par + oW[l], C * C, wb + static_cast<size_t>(l) * C * C, st);
        huv_launch::fno_tc_pack_zs(Za, rows, m, S, zs, st);
        if (!huv_launch::fno_tc_layer(B, S, m, v[l], wb + static_cast<size_t>(l) * C * C, tw_tab, zs, par + ob[l],
                                      l < L - 1 ? 1 : 0, z[l], v[l + 1], tc_err, st))
          throw Error(HUV_ERR_CUDA, "fno: tensor-core layer launch failed");
      } else {
        fno_layer_out<<<rgrid, 256, layer_out_smem(), st>>>(
            Za, v[l], par + oW[l], par + ob[l], S, m, twx, l < L - 1 ? 1 : 0, z[l], v[l + 1], rows);
      }
    }
    if (tc) {
      huv_launch::fno_tc_to_bf16(par + oQ1, P * C, q1b, st);
      if (!huv_launch::fno_tc_proj(B, S, v[L], q1b, par + ob1, par + oQ2, par + ob2, images ? images : out, tc_err, st))
        throw Error(HUV_ERR_CUDA, "fno: tensor-core projection launch failed");
    } else {
      fno_proj<<<pgrid(pix), 256, kProjSmem, st>>>(v[L], par + oQ1, par + ob1, par + oQ2, par + ob2, pix,
                                                   images ? images : out);
    }
    check_cuda(cudaGetLastError(), "fno forward");
  }

  // Backward from dout (device, [B][S][S]); accumulates into grad (zeroed
  // here) and writes the input gradient dmask when given.
  void backward(int B, const float* masks, const float* dOut, float* dmask, cudaStream_t st) {
    using namespace huv_dev;
    const size_t pix = static_cast<size_t>(B) * S * S;
    const int rows = B * S;
    const dim3 rgrid(std::min(rows, 4096));
    const dim3 ygrid((m * C + 63) / 64, B);
    check_cuda(cudaMemsetAsync(grad, 0, npar * 4, st), "memset grad");
    if (tc) {
      if (!huv_launch::fno_tc_proj_bwd(pix, v[L], par + oQ1, par + ob1, par + oQ2, dOut, dvA, grad + oQ1, grad + ob1,
                                       grad + oQ2, grad + ob2, tc_err, st))
        throw Error(HUV_ERR_CUDA, "fno: tensor-core projection backward launch failed");
    } else {
      fno_proj_bwd<<<std::min<size_t>((pix + 63) / 64, 148), 256, kProjBwdSmem, st>>>(
          v[L], par + oQ1, par + ob1, par + oQ2, pix, dOut, dvA, grad + oQ1, grad + ob1, grad + oQ2, grad + ob2);
    }
    float* dnext = dvA;
    float* dcur = dvB;
    for (int l = L - 1; l >= 0; --l) {
      if (tc) {
        if (!huv_launch::fno_tc_layer_bwd(pix, dnext, z[l], v[l], par + oW[l], l < L - 1 ? 1 : 0, dz, dcur,
                                          grad + oW[l], grad + ob[l], tc_err, st))
          throw Error(HUV_ERR_CUDA, "fno: tensor-core layer backward launch failed");
      } else {
        fno_layer_bwd<<<std::min(rows, 296), 256, kLayerBwdSmem, st>>>(
            dnext, z[l], v[l], par + oW[l], S, l < L - 1 ? 1 : 0, dz, dcur, grad + oW[l], grad + ob[l], rows);
      }
      fno_dft_x<float><<<rgrid, 256, kDftXSmem, st>>>(dz, S, m, twx, Xa, rows);
      fno_dft_y<false><<<ygrid, 256, 0, st>>>(Xa, S, C, m, twy, Y);
      fno_scale_modes<<<256, 256, 0, st>>>(Y, B, J, m, C, 1.f / (static_cast<float>(S) * S));
      fno_mix_bwd<<<modes, 256, static_cast<size_t>(2) * B * C * 8, st>>>(
          Xl[l], Y, reinterpret_cast<const float2*>(par + oR[l]), C, modes, B, dX,
          reinterpret_cast<float2*>(grad + oR[l]));
      fno_dft_y<true><<<dim3(S, B), 256, 0, st>>>(dX, S, C, m, twy, Za);
      fno_spec_to_dv<<<rgrid, 256, spec_smem(), st>>>(Za, S, m, twx, dcur, rows);
      std::swap(dnext, dcur);
    }
    fno_lift_bwd<<<1184, 256, 0, st>>>(masks, dnext, S, par + oWl, pix, grad + oWl, grad + obl, dmask);
    check_cuda(cudaGetLastError(), "fno backward");
  }

  // Synchronise and read (then clear) the flag a bounded wait of a
  // tensor-core kernel sets when it gives up; throws if it was set.
  void check_device_flag(cudaStream_t st) {
    check_cuda(cudaStreamSynchronize(st), "sync");
    if (!tc_err) return;
    int h = 0;
    check_cuda(cudaMemcpy(&h, tc_err, sizeof(int), cudaMemcpyDeviceToHost), "read fno error flag");
    if (h) {
      check_cuda(cudaMemset(tc_err, 0, sizeof(int)), "reset fno error flag");
      throw Error(HUV_ERR_DEVICE_TIMEOUT, "fno: a bounded device-side wait gave up; the results are not valid");
    }
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
      throw Error(HUV_ERR_UNSUPPORTED, "fno: the FNO kernels are specialised to width 64, projection 128");
    if (modes > 16)
      throw Error(HUV_ERR_UNSUPPORTED, "fno: the DFT tiles hold at most 16 retained modes per axis");
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
    f->check_device_flag(st);
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
    f->check_device_flag(st);
  });
}

huv_status huv_fno_device_status(void* fno, void* stream) {
  return fno_guard([&] {
    Fno* f = as_fno(fno);
    huv::check_cuda(cudaSetDevice(f->device), "cudaSetDevice");
    f->check_device_flag(static_cast<cudaStream_t>(stream));
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
    f->check_device_flag(static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
