// Pixel ILT on the device: batched cost, exact SOCS adjoint gradient and the
// CG (Polak-Ribiere+) / Armijo optimizer, for many masks at once.
//
// Follows crates/highuvlith-core/src/ilt.rs: m = sigmoid(beta theta)
// (538-542), t = a + (1 - a) m and M = FFT(t) (544-550), the resist-contour or
// image-fidelity data term (564-603), TV + binarisation regularisers
// (606-645), the adjoint of cost_and_gradient_with (667-738) and run_stage
// (755-866).  The forward fields are band-limited (kernels live on |m| <= h),
// so the adjoint needs only the band of FFT(G0 . E_k):
//     Q = sum_k conj(kappa_k) . band(FFT(G0 . E_k)),   dC/dm = 2 (1 - a) Re IFFT(Q)
// with E_k = IFFT(kappa_k . M) on the full grid and kappa_k the pre-scaled band
// kernels (sqrt(lambda_k) / N^2 folded in), G0 = (1 - phi) dC/dI + phi mean(dC/dI).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../engine.hpp"
#include "fft_block.cuh"
#include "fft_reg.cuh"

namespace huv_dev {

// ------------------------------------------------------------ elementwise
// t = a + (1 - a) sigmoid(beta theta) (the transmittance fed to the band FFT).
__global__ void ilt_transmittance(const float* __restrict__ theta, size_t n, float beta, float absorber,
                                  float* __restrict__ t) {
  // float4 body when both arrays are 16-byte aligned, scalar tail
  const bool vec = ((reinterpret_cast<uintptr_t>(theta) | reinterpret_cast<uintptr_t>(t)) & 15u) == 0;
  const size_t n4 = vec ? n / 4 : 0;
  const float4* th4 = reinterpret_cast<const float4*>(theta);
  float4* t4 = reinterpret_cast<float4*>(t);
  auto f = [&](float v) { return absorber + (1.f - absorber) / (1.f + __expf(-beta * v)); };
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float4 v = th4[i];
    t4[i] = make_float4(f(v.x), f(v.y), f(v.z), f(v.w));
  }
  for (size_t i = 4 * n4 + blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    t[i] = f(theta[i]);
}

__device__ __forceinline__ double block_sum_double(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;
}

// Data term on the image: cost parts sum r^2 and the image adjoint G = dC/dI.
// grid: (blocks_per_mask, masks); parts: [mask][block][2] = (sum r^2, sum G).
__global__ void ilt_data(const float* __restrict__ img, const float* __restrict__ target, size_t npix,
                         int kind, float thr, float steep, float dose, float* __restrict__ G,
                         double* __restrict__ parts) {
  __shared__ double red[32];
  const int mask = blockIdx.y;
  const float* im = img + mask * npix;
  const float* tg = target + mask * npix;
  float* g = G + mask * npix;
  const float inv_n = 1.f / static_cast<float>(npix);
  double sr = 0.0, sg = 0.0;
  auto term = [&](float I, float T, float& gv) {
    float r;
    if (kind == 0) {
      r = dose * I - T;
      gv = 2.f * r * dose * inv_n;
    } else {
      const float R = 1.f / (1.f + __expf(-steep * (dose * I - thr)));
      r = R - T;
      gv = 2.f * r * steep * R * (1.f - R) * dose * inv_n;
    }
    sr += static_cast<double>(r) * r;
    sg += gv;
  };
  // float4 body when the three planes are 16-byte aligned, scalar tail
  const bool vec =
      ((reinterpret_cast<uintptr_t>(im) | reinterpret_cast<uintptr_t>(tg) | reinterpret_cast<uintptr_t>(g)) & 15u) == 0;
  const size_t n4 = vec ? npix / 4 : 0;
  const float4* im4 = reinterpret_cast<const float4*>(im);
  const float4* tg4 = reinterpret_cast<const float4*>(tg);
  float4* g4 = reinterpret_cast<float4*>(g);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float4 I = im4[i], T = tg4[i];
    float4 o;
    term(I.x, T.x, o.x);
    term(I.y, T.y, o.y);
    term(I.z, T.z, o.z);
    term(I.w, T.w, o.w);
    g4[i] = o;
  }
  for (size_t i = 4 * n4 + blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npix;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    float gv;
    term(im[i], tg[i], gv);
    g[i] = gv;
  }
  const double a = block_sum_double(sr, red);
  const double b = block_sum_double(sg, red);
  if (threadIdx.x == 0) {
    double* p = parts + (static_cast<size_t>(mask) * gridDim.x + blockIdx.x) * 2;
    p[0] = a;
    p[1] = b;
  }
}

// Sum parts[mask][i][c] over i in order (deterministic). out[mask * ncomp + c].
__global__ void sum_parts(const double* __restrict__ parts, int nparts, int ncomp, int masks,
                          double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= masks * ncomp) return;
  const int mask = t / ncomp, c = t % ncomp;
  double s = 0.0;
  for (int i = 0; i < nparts; ++i) s += parts[(static_cast<size_t>(mask) * nparts + i) * ncomp + c];
  out[t] = s;
}

// Adjoint column pass.  CTA per (mask, strip of Wc columns): for every kernel
// k the column field E_k(., x) = IFFT_y of the band rows T_k(my, x), times
// G0(., x) = keep * G + add[mask], forward FFT_y, band rows [-hb, hb] kept:
// V[mask][k][my'][x].  grid: (L / Wc, masks).
__global__ void ilt_cols_adj(const float2* __restrict__ T, const float* __restrict__ G, int K, int hb, int lg,
                             int Wc, float keep, const double* __restrict__ sums, float flare_over_n,
                             float2* __restrict__ V, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int mask = blockIdx.y;
  const int x0 = blockIdx.x * Wc;
  float2* a = smem;
  float2* b = smem + (Wc << lg);
  float* g0 = reinterpret_cast<float*>(smem + 2 * (Wc << lg));  // [Wc][L]
  const float add = sums ? flare_over_n * static_cast<float>(sums[mask * 2 + 1]) : 0.f;
  const float* Gm = G + static_cast<size_t>(mask) * L * L;
  for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) {
    const int y = t / Wc, w = t - y * Wc;
    g0[(w << lg) + y] = keep * Gm[static_cast<size_t>(y) * L + x0 + w] + add;
  }
  const float2* Tm = T + static_cast<size_t>(mask) * K * B * L;
  float2* Vm = V + static_cast<size_t>(mask) * K * B * L;
  for (int k = 0; k < K; ++k) {
    for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) a[t] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int t = threadIdx.x; t < B * Wc; t += blockDim.x) {
      const int my = t / Wc, w = t - my * Wc;
      a[(w << lg) + ((my - hb) & (L - 1))] = Tm[((static_cast<size_t>(k) * B + my) << lg) + x0 + w];
    }
    __syncthreads();
    float2* r = block_fft<+1>(a, b, lg, Wc, tw);
    float2* o = (r == a) ? b : a;
    for (int t = threadIdx.x; t < (Wc << lg); t += blockDim.x) {
      const float s = g0[t];
      r[t] = make_float2(r[t].x * s, r[t].y * s);
    }
    __syncthreads();
    const float2* f = block_fft<-1>(r, o, lg, Wc, tw);
    for (int t = threadIdx.x; t < B * Wc; t += blockDim.x) {
      const int my = t / Wc, w = t - my * Wc;
      Vm[((static_cast<size_t>(k) * B + my) << lg) + x0 + w] = f[(w << lg) + ((my - hb) & (L - 1))];
    }
    __syncthreads();
  }
}

// ilt_cols_adj with register-radix passes (fft_reg.cuh), reading the x-major
// row transforms Tt[mask][k][x][my] of socs_rows_x.  CTA per (mask, S
// columns); each thread keeps G0 at its own (column, y) positions in
// registers across all kernels.  Per kernel: inverse FFT_y of the band column
// (P -> b0 [-> b1]), times G0, natural order into the other buffer, forward
// FFT_y, band rows [-hb, hb] kept: V[mask][k][my'][x] (the layout of
// ilt_rows_adj).  grid: (L / S, masks); shared: P (S B), two FFT buffers,
// a second band buffer P2 (S B).
template <int L, int S>
__global__ void __launch_bounds__(fr_threads(L, S), (L == 160 || L == 192) ? 3 : 1)
    ilt_cols_adj_xt(const float2* __restrict__ Tt, const float* __restrict__ G, int K, int hb, float keep,
                    const double* __restrict__ sums, float flare_over_n, float2* __restrict__ V,
                    const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  extern __shared__ float2 smem[];
  const int B = 2 * hb + 1;
  const int mask = blockIdx.y;
  const int x0 = blockIdx.x * S;
  const int t = threadIdx.x;
  float2* P = smem;  // [S][B]
  float2* b0 = smem + S * B;
  float2* b1 = b0 + fr_buf(L, S);
  // the inverse transform ends in `inv`, the weighted field goes to `oth`
  float2* inv = NP == 3 ? b1 : b0;
  float2* oth = NP == 3 ? b0 : b1;
  const float add = sums ? flare_over_n * static_cast<float>(sums[mask * 2 + 1]) : 0.f;
  const float* Gm = G + static_cast<size_t>(mask) * L * L;
  constexpr int NB = fr_per(L, S, NP - 1);  // last-pass butterflies per thread
  float g[NB * R];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int u = t + b * T;
    const int s = u % S, j = (u / S) % (L / R);  // guarded butterflies read a valid row
#pragma unroll
    for (int p = 0; p < R; ++p)
      g[b * R + p] = keep * Gm[static_cast<size_t>(j + p * (L / R)) * L + x0 + s] + add;
  }
  // kernel k's band columns arrive by cp.async in P[k & 1] while kernel
  // k - 1 is transformed
  float2* P2 = b1 + fr_buf(L, S);
  auto prefetch = [&](int k) {
    const float2* src = Tt + ((static_cast<size_t>(mask) * K + k) * L + x0) * B;
    float2* dst = (k & 1) ? P2 : P;
    for (int e = t; e < S * B; e += T) fr_cp_async8(dst + e, src + e);
    fr_cp_commit();
  };
  prefetch(0);
  for (int k = 0; k < K; ++k) {
    if (k + 1 < K) {
      prefetch(k + 1);  // its buffer was last read before the previous iteration's final barrier
      fr_cp_wait<1>();
    } else {
      fr_cp_wait<0>();
    }
    __syncthreads();
    fr_first_pass_band<L, S, +1>(t, (k & 1) ? P2 : P, B, hb, b0);
    __syncthreads();
    if constexpr (NP == 3) {
      fr_mid_pass<L, S, +1, 1>(t, b0, b1, tw);
      __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      if (t + b * T >= fr_nb(L, S, NP - 1)) break;
      int s, j;
      float2 v[R];
      fr_last_pass<L, S, +1>(t + b * T, inv, tw, s, j, v);
#pragma unroll
      for (int p = 0; p < R; ++p) {
        const float w = g[b * R + p];
        oth[fr_idx<S>(j + p * (L / R), s)] = make_float2(v[p].x * w, v[p].y * w);
      }
    }
    __syncthreads();
    if (t < fr_nb(L, S, 0)) {
      const int s = t % S, j = t / S;
      float2 v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = oth[fr_idx<S>(j + r * (L / 16), s)];
      fr_first_pass_vals<L, S, -1>(t, v, inv);
    }
    __syncthreads();
    const float2* cur = inv;
    if constexpr (NP == 3) {
      fr_mid_pass<L, S, -1, 1>(t, inv, oth, tw);
      __syncthreads();
      cur = oth;
    }
    float2* Vk = V + (static_cast<size_t>(mask) * K + k) * B * L + x0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      if (t + b * T >= fr_nb(L, S, NP - 1)) break;
      int s, j;
      float2 v[R];
      fr_last_pass<L, S, -1>(t + b * T, cur, tw, s, j, v);
#pragma unroll
      for (int p = 0; p < R; ++p) {
        const int idx = j + p * (L / R);
        const int mi = idx <= hb ? idx + hb : (idx >= L - hb ? idx - L + hb : -1);
        if (mi >= 0) Vk[static_cast<size_t>(mi) * L + s] = v[p];
      }
    }
    __syncthreads();
  }
}

// In place: Q <- its Hermitian part (Q(f) + conj(Q(-f))) / 2 on each mask's
// B x B band, so that IFFT(Q) is real and equals Re IFFT of the original.
__global__ void hermitian_part(float2* __restrict__ Q, int B, int masks) {
  const int half = (B * B + 1) / 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < half * masks; e += gridDim.x * blockDim.x) {
    const int mask = e / half, i = e - mask * half;
    float2* q = Q + static_cast<size_t>(mask) * B * B;
    const int j = B * B - 1 - i;
    const float2 a = q[i], c = q[j];
    const float2 h = make_float2(0.5f * (a.x + c.x), 0.5f * (a.y - c.y));
    q[i] = h;
    q[j] = make_float2(h.x, -h.y);
  }
}

// ilt_rows_adj with register-radix passes: CTA per (mask, band row my'),
// kernels taken S at a time as the S sequences of one transform (rows of V
// read straight from global memory in the first pass), forward FFT_x, and
// for each kept order conj(kappa_k) . value summed over the lanes that hold
// the same order (warp shuffles), then over the batches in registers.
// grid: (B, masks); shared: two FFT buffers.
template <int L, int S>
__global__ void __launch_bounds__(fr_threads(L, S), (L == 160 || L == 192) ? 3 : 1)
    ilt_rows_adj_xt(const float2* __restrict__ V, const float2* __restrict__ kband, int K, int hb,
                    float2* __restrict__ Q, const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  constexpr int NB = fr_per(L, S, NP - 1);
  constexpr int G = S < 32 ? S : 32;  // lanes of one order within a warp
  static_assert(32 % S == 0 || S % 32 == 0, "the lanes of one order must form a shuffle group");
  static_assert(fr_nb(L, S, NP - 1) % T == 0, "last-pass butterflies must fill every thread (warp-uniform)");
  extern __shared__ float2 smem[];
  const int B = 2 * hb + 1;
  const int mask = blockIdx.y, my = blockIdx.x;
  const int t = threadIdx.x;
  float2* b0 = smem;
  float2* b1 = b0 + fr_buf(L, S);
  float2 acc[NB * R];
#pragma unroll
  for (int i = 0; i < NB * R; ++i) acc[i] = make_float2(0.f, 0.f);
  for (int k0 = 0; k0 < K; k0 += S) {
    if (t < fr_nb(L, S, 0)) {
      const int s = t % S, j = t / S;
      const bool live = k0 + s < K;
      const float2* row = V + ((static_cast<size_t>(mask) * K + (live ? k0 + s : 0)) * B + my) * L + j;
      float2 v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = live ? row[r * (L / 16)] : make_float2(0.f, 0.f);
      fr_first_pass_vals<L, S, -1>(t, v, b0);
    }
    __syncthreads();
    const float2* cur = b0;
    if constexpr (NP == 3) {
      fr_mid_pass<L, S, -1, 1>(t, b0, b1, tw);
      __syncthreads();
      cur = b1;
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      int s, j;
      float2 v[R];
      fr_last_pass<L, S, -1>(t + b * T, cur, tw, s, j, v);
      const int k = k0 + s;
#pragma unroll
      for (int p = 0; p < R; ++p) {
        const int idx = j + p * (L / R);
        const int mi = idx <= hb ? idx + hb : (idx >= L - hb ? idx - L + hb : -1);
        float2 w = make_float2(0.f, 0.f);
        if (mi >= 0 && k < K) {
          const float2 u = kband[(static_cast<size_t>(k) * B + my) * B + mi];
          w = make_float2(u.x * v[p].x + u.y * v[p].y, u.x * v[p].y - u.y * v[p].x);  // conj(u) v
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
          w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
          w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
        }
        acc[b * R + p].x += w.x;
        acc[b * R + p].y += w.y;
      }
    }
    __syncthreads();
  }
  // with S > 32 an order's S lanes span S / 32 warps: they are summed in
  // shared memory (b0 is free after the final barrier)
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int u = t + b * T;
    const int s = u % S, j = u / S;
    if (s % G != 0) continue;
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const int idx = j + p * (L / R);
      const int mi = idx <= hb ? idx + hb : (idx >= L - hb ? idx - L + hb : -1);
      if (mi < 0) continue;
      if (S <= 32) {
        Q[(static_cast<size_t>(mask) * B + my) * B + mi] = acc[b * R + p];
      } else {
        b0[(s / G) * L + idx] = acc[b * R + p];
      }
    }
  }
  if constexpr (S > 32) {
    __syncthreads();
    for (int idx = t; idx < L; idx += T) {
      const int mi = idx <= hb ? idx + hb : (idx >= L - hb ? idx - L + hb : -1);
      if (mi < 0) continue;
      float2 a = make_float2(0.f, 0.f);
      for (int g = 0; g < S / G; ++g) a = fr_add(a, b0[g * L + idx]);
      Q[(static_cast<size_t>(mask) * B + my) * B + mi] = a;
    }
  }
}

// Adjoint row pass.  CTA per (mask, band row my'): forward FFT_x of every
// kernel's V row, band columns kept, Q(my', mx') = sum_k conj(kappa_k) . value.
// grid: (B, masks).
__global__ void ilt_rows_adj(const float2* __restrict__ V, const float2* __restrict__ kband, int K, int hb, int lg,
                             int S, float2* __restrict__ Q, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int mask = blockIdx.y, my = blockIdx.x;
  float2* a = smem;
  float2* b = smem + (S << lg);
  float2 acc = make_float2(0.f, 0.f);
  const float2* Vm = V + static_cast<size_t>(mask) * K * B * L;
  for (int k0 = 0; k0 < K; k0 += S) {
    const int ns = min(S, K - k0);
    for (int t = threadIdx.x; t < (S << lg); t += blockDim.x) {
      const int s = t >> lg, x = t & (L - 1);
      a[t] = s < ns ? Vm[((static_cast<size_t>(k0 + s) * B + my) << lg) + x] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* r = block_fft<-1>(a, b, lg, S, tw);
    if (threadIdx.x < B) {
      const int mx = threadIdx.x;
      for (int s = 0; s < ns; ++s) {
        const float2 v = r[(s << lg) + ((mx - hb) & (L - 1))];
        const float2 u = kband[(static_cast<size_t>(k0 + s) * B + my) * B + mx];
        // conj(u) * v
        acc.x += u.x * v.x + u.y * v.y;
        acc.y += u.x * v.y - u.y * v.x;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < B) Q[(static_cast<size_t>(mask) * B + my) * B + threadIdx.x] = acc;
}

// Regularisers and the chain rule: grad = (dC/dm + reg) * beta m (1 - m), with
// m = sigmoid(beta theta) recomputed; TV on forward differences (periodic).
// parts: [mask][block] reg cost.  dcdm may be NULL (cost only).
__global__ void ilt_finish(const float* __restrict__ theta, const float* __restrict__ dcdm, int n, float beta,
                           float tv_w, float tv_eps, float bin_w, float* __restrict__ grad,
                           double* __restrict__ parts) {
  __shared__ double red[32];
  const int mask = blockIdx.y;
  const size_t npix = static_cast<size_t>(n) * n;
  const float* th = theta + mask * npix;
  const float inv_n = 1.f / static_cast<float>(npix);
  auto M = [&](int i, int j) {
    i = (i + n) % n;
    j = (j + n) % n;
    return 1.f / (1.f + __expf(-beta * th[static_cast<size_t>(i) * n + j]));
  };
  double cost = 0.0;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < npix;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(p / n), j = static_cast<int>(p % n);
    const float m = M(i, j);
    float g = 0.f;
    if (tv_w > 0.f) {
      const float gx = M(i, j + 1) - m, gy = M(i + 1, j) - m;
      const float s = sqrtf(gx * gx + gy * gy + tv_eps * tv_eps);
      cost += static_cast<double>(tv_w) * (s - tv_eps) * inv_n;
      if (grad) {
        const float ml = M(i, j - 1), mu = M(i - 1, j);
        const float gxl = m - ml, gyl = M(i + 1, j - 1) - ml;
        const float sl = sqrtf(gxl * gxl + gyl * gyl + tv_eps * tv_eps);
        const float gxu = M(i - 1, j + 1) - mu, gyu = m - mu;
        const float su = sqrtf(gxu * gxu + gyu * gyu + tv_eps * tv_eps);
        g += tv_w * inv_n * (-(gx + gy) / s + gxl / sl + gyu / su);
      }
    }
    if (bin_w > 0.f) {
      cost += static_cast<double>(bin_w) * 4.0 * m * (1.0 - m) * inv_n;
      g += bin_w * 4.f * (1.f - 2.f * m) * inv_n;
    }
    if (grad) grad[mask * npix + p] = ((dcdm ? dcdm[mask * npix + p] : 0.f) + g) * beta * m * (1.f - m);
  }
  const double c = block_sum_double(cost, red);
  if (threadIdx.x == 0) parts[static_cast<size_t>(mask) * gridDim.x + blockIdx.x] = c;
}

// The same as ilt_finish for grids that are multiples of TS: a block takes a
// TS x TS tile, computes m = sigmoid(beta theta) once for the tile and its
// 1-pixel periodic halo in shared memory (instead of up to nine sigmoids per
// pixel), then each thread takes runs of 4 pixels of a row (16-byte loads of
// dC/dm and stores of the gradient), and writes its share of the regulariser
// cost to parts[mask][tile].  The thread's dC/dm runs and the halo's theta
// are all loaded before the first sigmoid, so both streams are in flight
// together (held to 64 registers, four blocks per SM: 1.597 -> 1.589 ms per
// C4 gradient; at three blocks per SM it was slower).  grid: ((n / TS)^2,
// masks), block 256.
template <int TS>
__global__ void __launch_bounds__(256, 4) ilt_finish_tiled(const float* __restrict__ theta,
                                                         const float* __restrict__ dcdm, int n, float beta,
                                                         float tv_w, float tv_eps, float bin_w,
                                                         float* __restrict__ grad, double* __restrict__ parts) {
  static_assert(TS % 4 == 0 && (TS * TS) % 1024 == 0, "tiles of whole 4-pixel runs, 256 threads");
  constexpr int NE = (TS + 2) * (TS + 2), NQ = (NE + 255) / 256;
  constexpr int RUNS = TS / 4;               // 4-pixel runs per row
  constexpr int ROWS_PER_PASS = 256 / RUNS;  // rows a pass of the block covers
  __shared__ float sm[TS + 2][TS + 3];
  __shared__ double red[32];
  const int mask = blockIdx.y;
  const size_t npix = static_cast<size_t>(n) * n;
  const int tiles_x = n / TS;
  const int ti = blockIdx.x / tiles_x, tj = blockIdx.x - ti * tiles_x;
  const float* th = theta + mask * npix;
  const float inv_n = 1.f / static_cast<float>(npix);
  constexpr int NPASS = TS / ROWS_PER_PASS;
  const int c4 = (threadIdx.x % RUNS) * 4, r0 = threadIdx.x / RUNS;
  float4 d4[NPASS];
#pragma unroll
  for (int q = 0; q < NPASS; ++q) {
    const size_t gp = mask * npix + static_cast<size_t>(ti * TS + r0 + q * ROWS_PER_PASS) * n + tj * TS + c4;
    d4[q] = dcdm ? *reinterpret_cast<const float4*>(dcdm + gp) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  float tv[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const int e = threadIdx.x + 256 * q;
    tv[q] = 0.f;
    if (e < NE) {
      const int r = e / (TS + 2), c = e - r * (TS + 2);
      int i = ti * TS - 1 + r, j = tj * TS - 1 + c;
      i = i < 0 ? i + n : (i >= n ? i - n : i);
      j = j < 0 ? j + n : (j >= n ? j - n : j);
      tv[q] = th[static_cast<size_t>(i) * n + j];
    }
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const int e = threadIdx.x + 256 * q;
    if (e < NE) {
      const int r = e / (TS + 2), c = e - r * (TS + 2);
      sm[r][c] = 1.f / (1.f + __expf(-beta * tv[q]));
    }
  }
  __syncthreads();
  // per-thread partials in FP32, the block sum in FP64
  float tv_part = 0.f, bin_part = 0.f;
  const float eps2 = tv_eps * tv_eps;
#pragma unroll
  for (int q = 0; q < NPASS; ++q) {
    const int r = r0 + q * ROWS_PER_PASS + 1;
    const size_t gp = mask * npix + static_cast<size_t>(ti * TS + r - 1) * n + tj * TS + c4;
    const float dv[4] = {d4[q].x, d4[q].y, d4[q].z, d4[q].w};
    float out[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = c4 + 1 + i;
      const float m = sm[r][c];
      float g = 0.f;
      if (tv_w > 0.f) {
        const float gx = sm[r][c + 1] - m, gy = sm[r + 1][c] - m;
        const float qv = gx * gx + gy * gy + eps2;
        const float iv = rsqrtf(qv);
        tv_part += qv * iv - tv_eps;
        if (grad) {
          const float ml = sm[r][c - 1], mu = sm[r - 1][c];
          const float gxl = m - ml, gyl = sm[r + 1][c - 1] - ml;
          const float il = rsqrtf(gxl * gxl + gyl * gyl + eps2);
          const float gxu = sm[r - 1][c + 1] - mu, gyu = m - mu;
          const float iu = rsqrtf(gxu * gxu + gyu * gyu + eps2);
          g += tv_w * inv_n * (-(gx + gy) * iv + gxl * il + gyu * iu);
        }
      }
      if (bin_w > 0.f) {
        bin_part += m * (1.f - m);
        g += bin_w * 4.f * (1.f - 2.f * m) * inv_n;
      }
      out[i] = (dv[i] + g) * beta * m * (1.f - m);
    }
    if (grad) *reinterpret_cast<float4*>(grad + gp) = make_float4(out[0], out[1], out[2], out[3]);
  }
  const double cost = (static_cast<double>(tv_w) * tv_part + 4.0 * static_cast<double>(bin_w) * bin_part) * inv_n;
  const double cs = block_sum_double(cost, red);
  if (threadIdx.x == 0) parts[static_cast<size_t>(mask) * gridDim.x + blockIdx.x] = cs;
}

// ------------------------------------------------------------ optimizer algebra
// Per-mask reductions over n elements: out[mask] = sum a*b (dot) or max |a|.
__global__ void batched_dot(const float* __restrict__ a, const float* __restrict__ b, size_t n,
                            double* __restrict__ parts) {
  __shared__ double red[32];
  const int mask = blockIdx.y;
  double s = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    s += static_cast<double>(a[mask * n + i]) * b[mask * n + i];
  const double t = block_sum_double(s, red);
  if (threadIdx.x == 0) parts[static_cast<size_t>(mask) * gridDim.x + blockIdx.x] = t;
}

__global__ void batched_maxabs(const float* __restrict__ a, size_t n, double* __restrict__ parts) {
  __shared__ double red[32];
  const int mask = blockIdx.y;
  float m = 0.f;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    m = fmaxf(m, fabsf(a[mask * n + i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
    parts[static_cast<size_t>(mask) * gridDim.x + blockIdx.x] = r;
  }
}

__global__ void max_parts(const double* __restrict__ parts, int nparts, int masks, double* __restrict__ out) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= masks) return;
  double r = 0.0;
  for (int i = 0; i < nparts; ++i) r = fmax(r, parts[static_cast<size_t>(m) * nparts + i]);
  out[m] = r;
}

// y[mask] = alpha[mask] * x[mask] + gamma[mask] * y[mask]   (per-mask scalars)
__global__ void batched_axpby(const float* __restrict__ x, float* __restrict__ y, size_t n,
                              const float* __restrict__ alpha, const float* __restrict__ gamma,
                              float* __restrict__ out) {
  const int mask = blockIdx.y;
  const float al = alpha[mask], ga = gamma[mask];
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[mask * n + i] = al * x[mask * n + i] + ga * y[mask * n + i];
}

__global__ void scale_inplace(float* __restrict__ x, size_t n, float s) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    x[i] *= s;
}

// parts[mask][block] = (max |a - b|, max |b|)
__global__ void err_parts(const float* __restrict__ a, const float* __restrict__ b, size_t n,
                          double* __restrict__ parts) {
  __shared__ float re[32], rb[32];
  const int mask = blockIdx.y;
  float e = 0.f, m = 0.f;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    e = fmaxf(e, fabsf(a[mask * n + i] - b[mask * n + i]));
    m = fmaxf(m, fabsf(b[mask * n + i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    re[threadIdx.x >> 5] = e;
    rb[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float E = 0.f, Mx = 0.f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
      E = fmaxf(E, re[w]);
      Mx = fmaxf(Mx, rb[w]);
    }
    double* p = parts + (static_cast<size_t>(mask) * gridDim.x + blockIdx.x) * 2;
    p[0] = E;
    p[1] = Mx;
  }
}

// cost[c] = weight * (sum r^2) / npix + reg[c]
__global__ void ilt_combine(const double* __restrict__ data, const double* __restrict__ reg, int masks, double w,
                            double inv_npix, double* __restrict__ cost) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < masks) cost[c] = w * data[2 * c] * inv_npix + reg[c];
}

// out[j] = alpha[j] * x[idx[j]] + gamma[j] * y[idx[j]]   (blocks of n floats)
__global__ void gather_axpby(const int* __restrict__ idx, const float* __restrict__ alpha,
                             const float* __restrict__ gamma, const float* __restrict__ x,
                             const float* __restrict__ y, size_t n, float* __restrict__ out) {
  const int j = blockIdx.y;
  const size_t m = static_cast<size_t>(idx[j]);
  const float al = alpha[j], ga = gamma[j];
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float xv = x ? x[m * n + i] : 0.f;
    const float yv = y ? y[m * n + i] : 0.f;
    out[j * n + i] = al * xv + ga * yv;
  }
}

// dst[idx[j]] = src[j]   (blocks of n floats)
__global__ void scatter_blocks(const int* __restrict__ idx, const float* __restrict__ src, size_t n,
                               float* __restrict__ dst) {
  const int j = blockIdx.y;
  const size_t m = static_cast<size_t>(idx[j]);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[m * n + i] = src[j * n + i];
}

}  // namespace huv_dev

// ================================================================== host
namespace huv_launch {
cudaError_t socs_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int lgm, int clips,
                      float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols(const float2* T, int K, int hb, int lgm, int clips, float keep, float flare,
                      const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
cudaError_t socs_rows_x(const float2* kband, float scale, const float2* Mband, int K, int hb, int L, int clips,
                        float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols_x(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                        const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
cudaError_t socs_cols_split(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                            const float* mean, void* split, const float2* tw, cudaStream_t st);

bool xt_ok(int L, int hb);

cudaError_t ilt_set_smem() {
  const int big = 200 * 1024;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_rows_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
  const int xt = huv_dev::kXtSmemMax;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<128, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<256, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<512, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<1024, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
#define HUV_ILT_XT(LL, SS)                                                                                   \
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_rows_adj_xt<LL, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt))) \
    return e;
  HUV_ILT_XT(128, 32) HUV_ILT_XT(160, 16) HUV_ILT_XT(192, 16) HUV_ILT_XT(256, 16) HUV_ILT_XT(512, 8)
  HUV_ILT_XT(1024, 4)
#undef HUV_ILT_XT
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<160, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::ilt_cols_adj_xt<192, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, xt)))
    return e;
  return cudaSuccess;
}

// Shared memory of ilt_cols_adj_xt on L points: two band-column buffers and
// two FFT buffers.
size_t ilt_adj_xt_smem(int L, int hb) {
  const int S = huv_dev::xt_S(L);
  return (2 * static_cast<size_t>(S) * (2 * hb + 1) + 2 * static_cast<size_t>(huv_dev::fr_buf(L, S))) *
         sizeof(float2);
}
}  // namespace huv_launch

namespace huv {

namespace {
size_t a256(size_t v) { return (v + 255) & ~size_t(255); }
int ilog2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
constexpr int kRedBlocks = 64;  // blocks per mask for reductions
}  // namespace

// Cost (and gradient when grad != nullptr) for `masks` masks on the device.
// cost_dev: masks doubles on the device.
//
// Every per-kernel field is evaluated on the coarse grid M > 4h (the
// smallest power of two, as for the image): the intensity is band-limited to
// 2h, so its exact N x N samples come from the M x M ones by band
// interpolation; the adjoint needs only the band h of G0 . E_k, which depends
// only on the band 2h of G0 = dC/dI, and the product of a band-2h and a
// band-h function is alias-free on M > 4h.  Hence
//   Q(f) = sum_k conj(kappa_k(f)) sum_{x in N^2} G0 E_k e^{-2 pi i f x / N}
//        = (N / M)^2 sum_k conj(kappa_k(f)) sum_{x' in M^2} G0' E_k e^{-2 pi i f x' / M},
// G0' the band-2h part of G0 sampled on the M grid.  Only the transmittance,
// the data term, G's band, dC/dm and the regularisers touch N x N.
void Engine::ilt_eval(const huv_ilt_params& p, int masks, const float* theta, const float* target, float* grad,
                      double* cost_dev, cudaStream_t st) {
  using namespace huv_dev;
  using namespace huv_launch;
  static std::atomic<uint64_t> smem_set{0};
  once_per_device(smem_set, [] { check_cuda(ilt_set_smem(), "cudaFuncSetAttribute(ilt)"); });
  DeviceSet& ds = device_set(p.defocus_nm == 0.0 ? 0.0 : p.defocus_nm);
  const int K = ds.K, hb = ds.hb, B = ds.B;
  const int h2 = 2 * hb, B2 = 2 * h2 + 1;
  const int lgn = ilog2i(n);
  // the smallest supported grid above 4h: 160 or 192 where the register-radix
  // forward and adjoint kernels serve it, else a power of two
  int M = choose_eval_grid(ds, 0, true);
  // the adjoint kernels have 160 and 192 instances but not 384
  if ((M & (M - 1)) != 0 && (M == 384 || ilt_adj_xt_smem(M, hb) > static_cast<size_t>(kXtSmemMax)))
    M = choose_eval_grid(ds, 0);
  const int lgm = ilog2i(M);  // rounded up where M is 160 or 192 (radix-4 paths are not used then)
  const bool coarse = M < n;
  const size_t npix = static_cast<size_t>(n) * n, mpix = static_cast<size_t>(M) * M;
  const float2* twn = twiddle_n(n);
  const float2* twm = twiddle_n(M);
  const float flare = ds.flare, keep = ds.keep;
  // Per-mask workspace.
  const size_t s_t = a256(sizeof(float) * npix);           // transmittance, then dC/dm
  const size_t s_x = a256(sizeof(float2) * n * B2);        // row transforms of N x N inputs (band <= 2h)
  const size_t s_m = a256(sizeof(float2) * B * B);
  const size_t s_mean = a256(sizeof(float) * (1 + (B2 + 3) / 4));
  const size_t s_T = a256(sizeof(float2) * static_cast<size_t>(K) * B * M);
  const size_t s_im = coarse ? a256(sizeof(float) * mpix) : 0;  // I on M, then G' on M
  const size_t s_c = coarse ? a256(sizeof(float2) * B2 * B2) : 0;
  const size_t s_x2 = coarse ? a256(sizeof(float2) * static_cast<size_t>(std::max(M, n)) * B2) : 0;
  // the image's interpolation from M to N: the separable tcgen05 GEMMs (as
  // the hybrid form) where they serve M, else the band transform of I_M and
  // N-point row and column syntheses
  const bool xt_fwd = M <= 1024 && xt_ok(M, hb) && ilt_adj_xt_smem(M, hb) <= static_cast<size_t>(kXtSmemMax);
  const bool sep = coarse && xt_fwd && separable_ok(ds, M);
  const size_t s_bi = sep ? a256(sizeof(uint16_t) * 2 * static_cast<size_t>(n) * M) : 0;
  const size_t s_img = a256(sizeof(float) * npix);         // image on N, then G
  const size_t s_V = grad ? a256(sizeof(float2) * static_cast<size_t>(K) * B * M) : 0;
  const size_t s_q = grad ? a256(sizeof(float2) * B * B) : 0;
  const size_t s_t2 = grad ? a256(sizeof(float2) * static_cast<size_t>(B) * n) : 0;
  const size_t s_parts = a256(sizeof(double) * kRedBlocks * 2);
  // 64 x 64 regulariser tiles where the grid allows (fewer, longer blocks),
  // else 32 x 32, else the untiled kernel
  const int tile = n % 64 == 0 ? 64 : (n % 32 == 0 ? 32 : 0);
  const bool tiled = tile > 0;
  const int reg_parts = tiled ? (n / tile) * (n / tile) : kRedBlocks;
  const size_t s_preg = a256(sizeof(double) * std::max(reg_parts, 2 * kRedBlocks));
  const size_t per = s_t + s_x + s_m + s_mean + s_T + s_im + s_c + s_x2 + s_img + s_V + s_q + s_t2 + 2 * s_parts +
                     s_preg + s_bi + a256(sizeof(double) * 4);
  const size_t budget = chunk_budget();
  const int chunk = balanced_chunk(static_cast<int>(std::max<size_t>(1, budget / per)), masks);
  char* base = static_cast<char*>(workspace(per * chunk + 4096));
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* q = base + off;
    off += bytes * chunk;
    return q;
  };
  float* tbuf = reinterpret_cast<float*>(take(s_t));
  float2* X = reinterpret_cast<float2*>(take(s_x));
  float2* Mb = reinterpret_cast<float2*>(take(s_m));
  float* mean = reinterpret_cast<float*>(take(s_mean));
  float2* T = reinterpret_cast<float2*>(take(s_T));
  float* IM = reinterpret_cast<float*>(take(s_im));
  float2* C = reinterpret_cast<float2*>(take(s_c));
  float2* X2 = reinterpret_cast<float2*>(take(s_x2));
  float* img = reinterpret_cast<float*>(take(s_img));
  float2* V = reinterpret_cast<float2*>(take(s_V));
  float2* Q = reinterpret_cast<float2*>(take(s_q));
  float2* T2 = reinterpret_cast<float2*>(take(s_t2));
  double* pdata = reinterpret_cast<double*>(take(s_parts));
  double* preg = reinterpret_cast<double*>(take(s_preg));
  double* sums = reinterpret_cast<double*>(take(s_parts));
  double* regsum = reinterpret_cast<double*>(take(a256(sizeof(double) * 4)));
  void* BI = sep ? static_cast<void*>(take(s_bi)) : nullptr;
  prof.begin(grad ? "ilt_cost_grad" : "ilt_cost", st);
  for (int c0 = 0; c0 < masks; c0 += chunk) {
    const int nc = std::min(chunk, masks - c0);
    const float* th = theta + npix * c0;
    const float* tg = target + npix * c0;
    ilt_transmittance<<<1184, 256, 0, st>>>(th, npix * nc, static_cast<float>(p.beta),
                                            static_cast<float>(p.absorber), tbuf);
    check_cuda(band_forward(tbuf, HUV_INPUT_RASTER_F32, n, lgn, hb, nc, X, Mb, nullptr, ds.W, mean, twn, st, nullptr, nullptr),
               "ilt band_forward");
    // fields of every kernel on the evaluation grid, the image on it, then on N x N
    // x-major row transforms (register-radix kernels) when the adjoint's
    // register-radix column pass fits too, else the [k][my][x] layout
    // (the ILT's grids are powers of two; ilt_cols_adj_xt has no 160 / 192 instance)
    // (the adjoint pair is instantiated up to 1024 points)
    const bool xt = xt_fwd;
    if (sep) {
      // I_M / interp_scale(mean) as FP16 split planes (in IM's bytes), then I_N = P I_M P^T
      check_cuda(socs_rows_x(ds.kband, 0.f, Mb, K, hb, M, nc, T, twm, st), "ilt socs_rows");
      check_cuda(socs_cols_split(T, K, hb, M, nc, keep, flare, mean, IM, twm, st), "ilt socs_cols");
      interp_separable(ds, M, nc, IM, mean, BI, img, st, false);
    } else if (xt) {
      check_cuda(socs_rows_x(ds.kband, 0.f, Mb, K, hb, M, nc, T, twm, st), "ilt socs_rows");
      check_cuda(socs_cols_x(T, K, hb, M, nc, keep, flare, mean, coarse ? IM : img, 0, twm, st), "ilt socs_cols");
    } else {
      check_cuda(socs_rows(ds.kband, 0.f, Mb, K, hb, lgm, nc, T, twm, st), "ilt socs_rows");
      check_cuda(socs_cols(T, K, hb, lgm, nc, keep, flare, mean, coarse ? IM : img, 0, twm, st), "ilt socs_cols");
    }
    if (coarse && !sep) {
      check_cuda(band_forward(IM, HUV_INPUT_RASTER_F32, M, lgm, h2, nc, X2, C, nullptr, nullptr, nullptr, twm, st, nullptr,
                              nullptr),
                 "ilt band(I)");
      const float scale = 1.0f / static_cast<float>(mpix);
      check_cuda(socs_rows_x(nullptr, scale, C, 1, h2, n, nc, X2, twn, st), "ilt interp rows");
      check_cuda(socs_cols_x(X2, 1, h2, n, nc, 1.f, 0.f, nullptr, img, 1, twn, st), "ilt interp cols");
    }
    ilt_data<<<dim3(kRedBlocks, nc), 256, 0, st>>>(img, tg, npix, p.cost_kind, static_cast<float>(p.threshold),
                                                   static_cast<float>(p.steepness), static_cast<float>(p.dose),
                                                   img, pdata);
    sum_parts<<<(nc * 2 + 127) / 128, 128, 0, st>>>(pdata, kRedBlocks, 2, nc, sums);
    float* dcdm = nullptr;
    if (grad) {
      // G' = the band-2h part of G = dC/dI, sampled on the evaluation grid
      const float* Gm = img;
      float grid_scale = 1.f;
      if (coarse) {
        check_cuda(band_forward(img, HUV_INPUT_RASTER_F32, n, lgn, h2, nc, X, C, nullptr, nullptr, nullptr, twn, st, nullptr,
                                nullptr),
                   "ilt band(G)");
        check_cuda(socs_rows_x(nullptr, 1.0f / static_cast<float>(npix), C, 1, h2, M, nc, X2, twm, st),
                   "ilt G rows");
        check_cuda(socs_cols_x(X2, 1, h2, M, nc, 1.f, 0.f, nullptr, IM, 1, twm, st), "ilt G cols");
        Gm = IM;
        grid_scale = static_cast<float>(static_cast<double>(npix) / static_cast<double>(mpix));
      }
      if (xt) {
        const dim3 ga(M / xt_S(M), nc);
        const size_t sm = ilt_adj_xt_smem(M, hb);
        const float fo = flare / static_cast<float>(npix);
        const dim3 gr(B, nc);
        const size_t smr = 2 * static_cast<size_t>(fr_buf(M, xt_S(M))) * sizeof(float2);
#define HUV_ILT_ADJ(LL, SS)                                                                 \
  ilt_cols_adj_xt<LL, SS><<<ga, 256, sm, st>>>(T, Gm, K, hb, keep, sums, fo, V, twm);    \
  ilt_rows_adj_xt<LL, SS><<<gr, 256, smr, st>>>(V, ds.kband, K, hb, Q, twm);
        switch (M) {
          case 128: HUV_ILT_ADJ(128, 32) break;
          case 160: HUV_ILT_ADJ(160, 16) break;
          case 192: HUV_ILT_ADJ(192, 16) break;
          case 256: HUV_ILT_ADJ(256, 16) break;
          case 512: HUV_ILT_ADJ(512, 8) break;
          case 1024: HUV_ILT_ADJ(1024, 4) break;
          default: throw Error(HUV_ERR_UNSUPPORTED, "ILT adjoint: no register-radix instance for this grid");
        }
#undef HUV_ILT_ADJ
      } else {
        const int Wc = fit_units(8, 2 * (sizeof(float2) << lgm) + (sizeof(float) << lgm));
        const size_t sm = 2 * (static_cast<size_t>(Wc) << lgm) * sizeof(float2) +
                          (static_cast<size_t>(Wc) << lgm) * sizeof(float);
        ilt_cols_adj<<<dim3(M / Wc, nc), 256, sm, st>>>(T, Gm, K, hb, lgm, Wc, keep, sums,
                                                        flare / static_cast<float>(npix), V, twm);
        const int S = fit_units(4, 2 * (sizeof(float2) << lgm));
        const size_t sm2 = 2 * (static_cast<size_t>(S) << lgm) * sizeof(float2);
        ilt_rows_adj<<<dim3(B, nc), 256, sm2, st>>>(V, ds.kband, K, hb, lgm, S, Q, twm);
      }
      const float scale = static_cast<float>(2.0 * (1.0 - p.absorber) * p.weight) * grid_scale;
      // Re IFFT(Q) = IFFT(Hermitian part of Q): a real synthesis, two
      // columns per transform on the register-radix path
      hermitian_part<<<(nc * ((B * B + 1) / 2) + 255) / 256, 256, 0, st>>>(Q, B, nc);
      check_cuda(socs_rows_x(nullptr, scale, Q, 1, hb, n, nc, T2, twn, st), "ilt grad rows");
      dcdm = tbuf;  // the transmittance is no longer needed
      check_cuda(socs_cols_x(T2, 1, hb, n, nc, 1.f, 0.f, nullptr, dcdm, 1, twn, st), "ilt grad cols");
    }
    if (tile == 64)
      ilt_finish_tiled<64><<<dim3(reg_parts, nc), 256, 0, st>>>(
          th, dcdm, n, static_cast<float>(p.beta), static_cast<float>(p.tv_weight),
          static_cast<float>(p.tv_epsilon), static_cast<float>(p.binarization_weight),
          grad ? grad + npix * c0 : nullptr, preg);
    else if (tiled)
      ilt_finish_tiled<32><<<dim3(reg_parts, nc), 256, 0, st>>>(
          th, dcdm, n, static_cast<float>(p.beta), static_cast<float>(p.tv_weight),
          static_cast<float>(p.tv_epsilon), static_cast<float>(p.binarization_weight),
          grad ? grad + npix * c0 : nullptr, preg);
    else
      ilt_finish<<<dim3(kRedBlocks, nc), 256, 0, st>>>(th, dcdm, n, static_cast<float>(p.beta),
                                                       static_cast<float>(p.tv_weight),
                                                       static_cast<float>(p.tv_epsilon),
                                                       static_cast<float>(p.binarization_weight),
                                                       grad ? grad + npix * c0 : nullptr, preg);
    sum_parts<<<(nc + 127) / 128, 128, 0, st>>>(preg, reg_parts, 1, nc, regsum);
    ilt_combine<<<(nc + 127) / 128, 128, 0, st>>>(sums, regsum, nc, p.weight, 1.0 / static_cast<double>(npix),
                                                  cost_dev + c0);
    check_cuda(cudaGetLastError(), "ilt kernels");
    prof.launches += (grad ? 17 : 10) + (coarse ? (grad ? 9 : 4) : 0) - (sep ? 2 : 0);
  }
  prof.end(st);
}

// Surrogate-based ILT cost and gradient: the transmittance's image comes
// from `sur`, its adjoint through the surrogate's input gradient; data term,
// regularisers and chain rule as in the exact path.
void Engine::ilt_eval_surrogate(Surrogate* sur, const huv_ilt_params& p, int masks, const float* theta,
                                const float* target, float* grad, double* cost_dev, cudaStream_t st) {
  using namespace huv_dev;
  const size_t npix = static_cast<size_t>(n) * n;
  const size_t per = 3 * ((sizeof(float) * npix + 255) & ~size_t(255)) + 3 * 256 * 8 * 2;
  char* base = static_cast<char*>(workspace(per * masks + 4096));
  float* tbuf = reinterpret_cast<float*>(base);
  float* img = tbuf + npix * masks;
  float* dt = img + npix * masks;
  double* pdata = reinterpret_cast<double*>(dt + npix * masks);
  double* preg = pdata + static_cast<size_t>(masks) * kRedBlocks * 2;
  double* sums = preg + static_cast<size_t>(masks) * kRedBlocks;
  double* regsum = sums + 2 * masks;
  ilt_transmittance<<<1184, 256, 0, st>>>(theta, npix * masks, static_cast<float>(p.beta),
                                          static_cast<float>(p.absorber), tbuf);
  sur->forward(masks, tbuf, img, st);
  ilt_data<<<dim3(kRedBlocks, masks), 256, 0, st>>>(img, target, npix, p.cost_kind, static_cast<float>(p.threshold),
                                                    static_cast<float>(p.steepness), static_cast<float>(p.dose), img,
                                                    pdata);
  sum_parts<<<(masks * 2 + 127) / 128, 128, 0, st>>>(pdata, kRedBlocks, 2, masks, sums);
  float* dcdm = nullptr;
  if (grad) {
    sur->input_grad(masks, tbuf, img, dt, st);  // img now holds G = dC/dI
    // dC/dm = weight (1 - a) dC/dt
    const float sc = static_cast<float>(p.weight * (1.0 - p.absorber));
    scale_inplace<<<1184, 256, 0, st>>>(dt, npix * masks, sc);
    dcdm = dt;
  }
  ilt_finish<<<dim3(kRedBlocks, masks), 256, 0, st>>>(theta, dcdm, n, static_cast<float>(p.beta),
                                                      static_cast<float>(p.tv_weight), static_cast<float>(p.tv_epsilon),
                                                      static_cast<float>(p.binarization_weight), grad, preg);
  sum_parts<<<(masks + 127) / 128, 128, 0, st>>>(preg, kRedBlocks, 1, masks, regsum);
  ilt_combine<<<(masks + 127) / 128, 128, 0, st>>>(sums, regsum, masks, p.weight, 1.0 / static_cast<double>(npix),
                                                   cost_dev);
  check_cuda(cudaGetLastError(), "ilt surrogate kernels");
}

std::vector<double> Engine::surrogate_error(Surrogate* sur, const huv_ilt_params& p, int masks, const float* theta,
                                            cudaStream_t st) {
  using namespace huv_dev;
  const size_t npix = static_cast<size_t>(n) * n;
  float *t = nullptr, *a = nullptr, *b = nullptr;
  double* parts = nullptr;
  check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&t), sizeof(float) * npix * masks * 3, st), "cudaMallocAsync");
  check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&parts), sizeof(double) * masks * kRedBlocks * 2, st),
             "cudaMallocAsync");
  a = t + npix * masks;
  b = a + npix * masks;
  ilt_transmittance<<<1184, 256, 0, st>>>(theta, npix * masks, static_cast<float>(p.beta),
                                          static_cast<float>(p.absorber), t);
  sur->forward(masks, t, a, st);
  huv_batch bt{};
  bt.n_clips = masks;
  bt.input_kind = HUV_INPUT_RASTER_F32;
  bt.input = t;
  bt.pixel_transfer = 0;
  bt.defocus_nm = p.defocus_nm;
  bt.form = HUV_FORM_AUTO;
  DeviceSet& ds = device_set(p.defocus_nm);
  int M = choose_eval_grid(ds, 0);
  if (tc_supported(ds, std::max(M, 128)) && n >= 128)
    run_tc_form(bt, ds, std::max(M, 128), b, st, 0, nullptr, kTcCoreFftField);  // the hybrid form
  else
    run_fft_form(bt, ds, M, b, st);
  // per mask: max |a - b| and max |b|
  err_parts<<<dim3(kRedBlocks, masks), 256, 0, st>>>(a, b, npix, parts);
  std::vector<double> h(static_cast<size_t>(masks) * kRedBlocks * 2);
  check_cuda(cudaMemcpyAsync(h.data(), parts, h.size() * 8, cudaMemcpyDeviceToHost, st), "D2H err");
  check_cuda(cudaFreeAsync(t, st), "cudaFreeAsync");
  check_cuda(cudaFreeAsync(parts, st), "cudaFreeAsync");
  check_cuda(cudaStreamSynchronize(st), "sync");
  std::vector<double> out(masks);
  for (int m2 = 0; m2 < masks; ++m2) {
    double e = 0, r = 0;
    for (int i = 0; i < kRedBlocks; ++i) {
      e = std::max(e, h[(static_cast<size_t>(m2) * kRedBlocks + i) * 2]);
      r = std::max(r, h[(static_cast<size_t>(m2) * kRedBlocks + i) * 2 + 1]);
    }
    out[m2] = r > 0 ? e / r : 0.0;
  }
  return out;
}

}  // namespace huv

// ------------------------------------------------------------ optimizer
namespace huv {

namespace {

}  // namespace

void IltOptState::DevVec::ensure(size_t b) {
  if (b <= bytes) return;
  cudaFree(p);
  p = nullptr;
  bytes = 0;
  check_cuda(cudaMalloc(&p, b), "cudaMalloc(ilt state)");
  bytes = b;
}

void IltOptState::release() {
  for (DevVec* v : {&grad, &dir, &gnew, &trial, &tgt, &gold, &cost_d, &parts, &dots, &alpha, &gamma, &idx}) {
    cudaFree(v->p);
    v->p = nullptr;
    v->bytes = 0;
  }
}

void Engine::ilt_optimize(const huv_ilt_params& p, const huv_ilt_opt& o, int masks, float* theta, const float* target,
                          double* final_cost, int* iterations, double* history, cudaStream_t st, Surrogate* sur,
                          int judge_every, double error_bound, SurrogateReport* report) {
  using namespace huv_dev;
  const size_t npix = static_cast<size_t>(n) * n;
  const size_t blk = sizeof(float) * npix;
  // optimizer state kept by the engine across calls (grown, never shrunk)
  IltOptState& S = ilt_state;
  auto& grad = S.grad;
  auto& dir = S.dir;
  auto& gnew = S.gnew;
  auto& trial = S.trial;
  auto& tgt = S.tgt;
  auto& gold = S.gold;
  auto& cost_d = S.cost_d;
  auto& parts = S.parts;
  auto& dots = S.dots;
  auto& alpha = S.alpha;
  auto& gamma = S.gamma;
  auto& idx = S.idx;
  grad.ensure(blk * masks);
  dir.ensure(blk * masks);
  gnew.ensure(blk * masks);
  trial.ensure(blk * masks);
  tgt.ensure(blk * masks);
  gold.ensure(blk * masks);
  cost_d.ensure(sizeof(double) * masks);
  parts.ensure(sizeof(double) * masks * kRedBlocks);
  dots.ensure(sizeof(double) * masks);
  alpha.ensure(sizeof(float) * masks);
  gamma.ensure(sizeof(float) * masks);
  idx.ensure(sizeof(int) * masks);
  const int max_it = o.max_iterations;
  const double lr = o.learning_rate, tol = o.convergence_tol;
  const int threads = 256;

  auto upload = [&](IltOptState::DevVec& v, const void* h, size_t b) {
    check_cuda(cudaMemcpyAsync(v.p, h, b, cudaMemcpyHostToDevice, st), "upload ilt scalars");
  };
  auto fetch = [&](const IltOptState::DevVec& v, void* h, size_t b) {
    check_cuda(cudaMemcpyAsync(h, v.p, b, cudaMemcpyDeviceToHost, st), "fetch ilt scalars");
    check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize(ilt)");
  };
  // per-mask dot products of compact blocks a[j], b[j], j < count
  auto dot = [&](const float* a, const float* b, int count) {
    batched_dot<<<dim3(kRedBlocks, count), threads, 0, st>>>(a, b, npix, parts.as<double>());
    sum_parts<<<(count + 127) / 128, 128, 0, st>>>(parts.as<double>(), kRedBlocks, 1, count, dots.as<double>());
    std::vector<double> h(count);
    fetch(dots, h.data(), sizeof(double) * count);
    prof.launches += 2;
    return h;
  };
  auto maxabs = [&](const float* a, int count) {
    batched_maxabs<<<dim3(kRedBlocks, count), threads, 0, st>>>(a, npix, parts.as<double>());
    max_parts<<<(count + 127) / 128, 128, 0, st>>>(parts.as<double>(), kRedBlocks, count, dots.as<double>());
    std::vector<double> h(count);
    fetch(dots, h.data(), sizeof(double) * count);
    prof.launches += 2;
    return h;
  };
  // out[j] = al[j] x[ix[j]] + ga[j] y[ix[j]]
  auto gaxpby = [&](const std::vector<int>& ix, const std::vector<float>& al, const std::vector<float>& ga,
                    const float* x, const float* y, float* out) {
    const int c = static_cast<int>(ix.size());
    if (!c) return;
    upload(idx, ix.data(), sizeof(int) * c);
    upload(alpha, al.data(), sizeof(float) * c);
    upload(gamma, ga.data(), sizeof(float) * c);
    gather_axpby<<<dim3(256, c), threads, 0, st>>>(idx.as<int>(), alpha.as<float>(), gamma.as<float>(), x, y, npix,
                                                   out);
    prof.launches += 1;
  };
  auto scatter = [&](const std::vector<int>& ix, const float* src, float* dst) {
    const int c = static_cast<int>(ix.size());
    if (!c) return;
    upload(idx, ix.data(), sizeof(int) * c);
    scatter_blocks<<<dim3(256, c), threads, 0, st>>>(idx.as<int>(), src, npix, dst);
    prof.launches += 1;
  };
  bool use_sur = sur != nullptr;
  auto eval = [&](const float* th, const float* tg, int count, float* g) {
    if (use_sur)
      ilt_eval_surrogate(sur, p, count, th, tg, g, cost_d.as<double>(), st);
    else
      ilt_eval(p, count, th, tg, g, cost_d.as<double>(), st);
    std::vector<double> h(count);
    fetch(cost_d, h.data(), sizeof(double) * count);
    return h;
  };
  auto ones = [](size_t c, float v) { return std::vector<float>(c, v); };

  std::vector<int> all(masks);
  for (int m = 0; m < masks; ++m) all[m] = m;
  std::vector<double> cost = eval(theta, target, masks, grad.as<float>());
  std::vector<std::vector<double>> hist(masks);
  for (int m = 0; m < masks; ++m) hist[m].push_back(cost[m]);
  gaxpby(all, ones(masks, -1.f), ones(masks, 0.f), grad.as<float>(), nullptr, dir.as<float>());
  std::vector<double> step(masks, lr);
  std::vector<int> small(masks, 0), its(masks, 0);
  std::vector<char> done(masks, 0);
  for (int it = 0; it < max_it; ++it) {
    std::vector<int> act;
    for (int m = 0; m < masks; ++m)
      if (!done[m]) act.push_back(m);
    if (use_sur && judge_every > 0 && ((it > 0 && it % judge_every == 0) || act.empty())) {
      // Exact SOCS re-images every mask (also when the surrogate run has
      // stopped) and judges the surrogate; past the bound it takes over for
      // all masks, stopped ones included.
      act = all;
      const int ac0 = masks;
      gaxpby(act, ones(ac0, 1.f), ones(ac0, 0.f), theta, nullptr, trial.as<float>());
      const std::vector<double> err = surrogate_error(sur, p, ac0, trial.as<float>(), st);
      const double worst = *std::max_element(err.begin(), err.end());
      if (report) report->judge_errors.push_back(worst);
      if (worst > error_bound) {
        // Takeover: exact costs and gradients from here on.
        use_sur = false;
        if (report) report->takeover_iteration = it;
        gaxpby(act, ones(ac0, 1.f), ones(ac0, 0.f), target, nullptr, tgt.as<float>());
        const std::vector<double> ce = eval(trial.as<float>(), tgt.as<float>(), ac0, gnew.as<float>());
        scatter(act, gnew.as<float>(), grad.as<float>());
        gaxpby(act, ones(ac0, -1.f), ones(ac0, 0.f), grad.as<float>(), nullptr, gnew.as<float>());
        scatter(act, gnew.as<float>(), dir.as<float>());
        for (int j = 0; j < ac0; ++j) {
          cost[act[j]] = ce[j];
          small[act[j]] = 0;
          done[act[j]] = 0;
        }
      }
      if (use_sur) {
        act.clear();
        for (int m = 0; m < masks; ++m)
          if (!done[m]) act.push_back(m);
      }
    }
    if (act.empty()) break;
    if (report) (use_sur ? report->surrogate_iterations : report->exact_iterations) += 1;
    std::vector<double> acc_cost(masks, 0.0), acc_s(masks, 0.0);
    std::vector<char> accepted(masks, 0);
    std::vector<int> attempt_set = act;
    for (int attempt = 0; attempt < 2 && !attempt_set.empty(); ++attempt) {
      // direction data for the attempt set (gathered into `trial` compactly)
      const int c = static_cast<int>(attempt_set.size());
      gaxpby(attempt_set, ones(c, 1.f), ones(c, 0.f), dir.as<float>(), nullptr, trial.as<float>());
      gaxpby(attempt_set, ones(c, 1.f), ones(c, 0.f), grad.as<float>(), nullptr, gold.as<float>());
      const std::vector<double> dmax = maxabs(trial.as<float>(), c);
      const std::vector<double> gd = dot(gold.as<float>(), trial.as<float>(), c);
      std::vector<int> search, restart;
      std::vector<double> slope(masks, 0.0), dm(masks, 0.0);
      for (int j = 0; j < c; ++j) {
        const int m = attempt_set[j];
        if (dmax[j] == 0.0) continue;  // no direction: the mask stops
        dm[m] = dmax[j];
        slope[m] = gd[j] / dmax[j];
        if (slope[m] >= 0.0)
          restart.push_back(m);
        else
          search.push_back(m);
      }
      // Armijo backtracking for `search`.
      std::vector<double> s(masks);
      for (int m : search) s[m] = step[m];
      std::vector<int> pending = search;
      for (int bt = 0; bt < 25 && !pending.empty(); ++bt) {
        const int pc = static_cast<int>(pending.size());
        std::vector<float> al(pc), ga(pc, 1.f);
        for (int j = 0; j < pc; ++j) al[j] = static_cast<float>(s[pending[j]] / dm[pending[j]]);
        gaxpby(pending, al, ga, dir.as<float>(), theta, trial.as<float>());
        gaxpby(pending, ones(pc, 1.f), ones(pc, 0.f), target, nullptr, tgt.as<float>());
        const std::vector<double> ct = eval(trial.as<float>(), tgt.as<float>(), pc, nullptr);
        std::vector<int> ok_j, ok_m, next;
        for (int j = 0; j < pc; ++j) {
          const int m = pending[j];
          if (std::isfinite(ct[j]) && ct[j] <= cost[m] + 1e-4 * s[m] * slope[m]) {
            accepted[m] = 1;
            acc_cost[m] = ct[j];
            acc_s[m] = s[m];
            ok_j.push_back(j);
            ok_m.push_back(m);
          } else {
            s[m] *= 0.5;
            next.push_back(m);
          }
        }
        // accepted trials become the new theta
        if (!ok_j.empty()) {
          std::vector<float> one(ok_j.size(), 1.f), zero(ok_j.size(), 0.f);
          gaxpby(ok_j, one, zero, trial.as<float>(), nullptr, gnew.as<float>());
          scatter(ok_m, gnew.as<float>(), theta);
        }
        pending = next;
      }
      // next attempt: restarts, and (first attempt only) failed searches, along -grad
      std::vector<int> nxt = restart;
      if (attempt == 0)
        for (int m : search)
          if (!accepted[m]) nxt.push_back(m);
      if (!nxt.empty()) {
        const int nc = static_cast<int>(nxt.size());
        gaxpby(nxt, ones(nc, -1.f), ones(nc, 0.f), grad.as<float>(), nullptr, gnew.as<float>());
        scatter(nxt, gnew.as<float>(), dir.as<float>());
      }
      attempt_set = attempt == 0 ? nxt : std::vector<int>();
    }
    std::vector<int> acc;
    for (int m : act) {
      if (accepted[m])
        acc.push_back(m);
      else
        done[m] = 1;  // line search failed (or no direction)
    }
    if (acc.empty()) break;
    // gradient at the accepted points (compact), then the CG direction
    const int ac = static_cast<int>(acc.size());
    gaxpby(acc, ones(ac, 1.f), ones(ac, 0.f), theta, nullptr, trial.as<float>());
    gaxpby(acc, ones(ac, 1.f), ones(ac, 0.f), target, nullptr, tgt.as<float>());
    const std::vector<double> cn = eval(trial.as<float>(), tgt.as<float>(), ac, gnew.as<float>());
    gaxpby(acc, ones(ac, 1.f), ones(ac, 0.f), grad.as<float>(), nullptr, gold.as<float>());
    const std::vector<double> gg = dot(gold.as<float>(), gold.as<float>(), ac);
    const std::vector<double> nn = dot(gnew.as<float>(), gnew.as<float>(), ac);
    const std::vector<double> ng = dot(gnew.as<float>(), gold.as<float>(), ac);
    std::vector<float> al(ac, -1.f), be(ac);
    for (int j = 0; j < ac; ++j) be[j] = static_cast<float>(gg[j] > 0 ? std::max((nn[j] - ng[j]) / gg[j], 0.0) : 0.0);
    // dir = -gnew + beta * dir  (compact gnew with index j; dir with index m): do it in two steps
    gaxpby(acc, ones(ac, 0.f), be, dir.as<float>(), dir.as<float>(), gold.as<float>());  // gold[j] = beta dir[m]
    {
      // gold[j] -= gnew[j]; with identity indices
      std::vector<int> id(ac);
      for (int j = 0; j < ac; ++j) id[j] = j;
      gaxpby(id, ones(ac, -1.f), ones(ac, 1.f), gnew.as<float>(), gold.as<float>(), trial.as<float>());
      scatter(acc, trial.as<float>(), dir.as<float>());
      scatter(acc, gnew.as<float>(), grad.as<float>());
    }
    for (int j = 0; j < ac; ++j) {
      const int m = acc[j];
      const double prev = cost[m];
      cost[m] = cn[j];
      hist[m].push_back(cost[m]);
      ++its[m];
      step[m] = std::min(acc_s[m] * 1.5, 10.0 * lr);
      const double rel = prev > 0 ? (prev - cost[m]) / prev : 0.0;
      small[m] = rel < tol ? small[m] + 1 : 0;
      if (small[m] >= 3 || cost[m] == 0.0) done[m] = 1;
    }
  }
  if (sur && use_sur) {
    // Report exact costs at the final masks.
    use_sur = false;
    const std::vector<double> ce = eval(theta, target, masks, nullptr);
    for (int m = 0; m < masks; ++m) cost[m] = ce[m];
  }
  for (int m = 0; m < masks; ++m) {
    if (final_cost) final_cost[m] = cost[m];
    if (iterations) iterations[m] = its[m];
    if (history)
      for (int i = 0; i <= max_it; ++i)
        history[static_cast<size_t>(m) * (max_it + 1) + i] =
            i < static_cast<int>(hist[m].size()) ? hist[m][i] : std::nan("");
  }
}

}  // namespace huv
