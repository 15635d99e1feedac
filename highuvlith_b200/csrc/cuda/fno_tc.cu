// tcgen05 channel GEMMs of the FNO forward pass (grids of at least 128).
//
// The pointwise layer and the projection head are contractions over the 64
// channels of every pixel: [pixels x 64] x [64 x N].  Pixels are tiled by
// 128 (one tile never crosses an image row when the grid is >= 128); the
// channels-last BF16 activations of a tile are one 128 x 128-byte TMA box
// (128B swizzle, K-major), the weights are resident in shared memory.
//
// MODE 0 (layer l): D[p][o] = sum_i v[p][i] W[o][i]
//                           + sum_kk Tw[x(p)][kk] Zs[row(p)][o][kk]
// where the second term is the layer's inverse x-DFT of the retained modes
// (Tw[x][2kx] = cos, Tw[x][2kx+1] = sin of 2 pi kx x / S; Zs = (w_kx / S^2)
// (Re Z, -Im Z) per image row), folded in as a second K block.  Epilogue:
// z = D + b, z stored (BF16) for the backward pass, v_next = GELU(z).
// MODE 1 (projection): D[p][j] = sum_i v[p][i] Q1[j][i], j < 128; epilogue
// out[p] = sum_j Q2[j] GELU(D[p][j] + b1[j]) + b2, one pixel per thread.
//
// Warp roles: 0 TMA producer (no multicast), 1 MMA issuer (one thread),
// 2..5 epilogue (one tensor-memory lane quadrant each).  Two shared-memory
// stages, tensor memory double-buffered, two CTAs per SM.  Every mbarrier wait is bounded
// (2 s); a timeout sets *err and unwinds.  Operands BF16, accumulation FP32.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../engine.hpp"
#include "tc_ptx.cuh"

namespace huv_dev {

constexpr int kFnoStages = 2;  // two stages keep two CTAs (8 epilogue warps) per SM
constexpr uint64_t kFnoWaitNs = 2000000000ull;
constexpr uint32_t kTile = 128 * 128;  // 128 rows x 64 bf16

struct FnoTcParams {
  int tiles;          // 128-pixel tiles
  int S;              // grid side
  int kk_steps;       // MODE 0: 16-wide K steps of the spectral block (ceil(2m / 16))
  const float* bias;  // MODE 0: b[64]; MODE 1: b1[128]
  const float* q2;    // MODE 1: Q2[128]
  const float* b2;    // MODE 1: b2[1]
  __nv_bfloat16* zsave;
  __nv_bfloat16* vnext;
  int act;            // MODE 0: GELU on v_next
  float* out;         // MODE 1
  int* err;
};

__device__ __forceinline__ float tc_gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }

template <int MODE>
__global__ void __launch_bounds__(192, 2)
    fno_tc_pw(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmW,
              const __grid_constant__ CUtensorMap tmTw, const __grid_constant__ CUtensorMap tmZ, FnoTcParams p) {
  constexpr int N = MODE == 0 ? 64 : 128;
  constexpr uint32_t kWBytes = N * 128;                              // resident weights
  constexpr uint32_t kStage = MODE == 0 ? 2 * kTile + 64 * 128 : kTile;  // v (+ twiddles + Zs)
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* sW = base;
  uint8_t* sS = base + kWBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sS + kFnoStages * kStage);
  uint64_t* full = bars;
  uint64_t* empty = bars + kFnoStages;
  uint64_t* w_full = bars + 2 * kFnoStages;
  uint64_t* tfull = bars + 2 * kFnoStages + 1;
  uint64_t* tempty = bars + 2 * kFnoStages + 3;
  uint64_t* done = bars + 2 * kFnoStages + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kFnoStages + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t kTmemCols = 2 * N <= 128 ? 128 : 256;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kFnoStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(w_full, 1);
    mbar_init(&tfull[0], 1);
    mbar_init(&tfull[1], 1);
    mbar_init(&tempty[0], 4);
    mbar_init(&tempty[1], 4);
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  auto fail = [&](int code) {
    *abort_flag = 1;
    if (p.err) atomicExch(p.err, code);
  };
  const int SS = p.S * p.S;

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&tmV);
      prefetch_tmap(&tmW);
      mbar_arrive_expect_tx(w_full, kWBytes);
      tma_load_2d(sW, &tmW, 0, 0, w_full);
      int it = 0;
      for (int t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x, ++it) {
        const int s = it % kFnoStages;
        if (!mbar_wait(&empty[s], ((it / kFnoStages) & 1) ^ 1, kFnoWaitNs)) {
          fail(11);
          break;
        }
        uint8_t* st = sS + s * kStage;
        const int p0 = t * 128;
        mbar_arrive_expect_tx(&full[s], kStage);
        tma_load_2d(st, &tmV, 0, p0, &full[s]);
        if (MODE == 0) {
          const int b = p0 / SS, rem = p0 - b * SS, y = rem / p.S, x0 = rem - y * p.S;
          tma_load_2d(st + kTile, &tmTw, 0, x0, &full[s]);
          tma_load_2d(st + 2 * kTile, &tmZ, 0, (b * p.S + y) * 64, &full[s]);
        }
      }
      // every load issued lands before the CTA may exit
      mbar_wait(w_full, 0, kFnoWaitNs);
      for (int q = (it > kFnoStages ? it - kFnoStages : 0); q < it; ++q)
        mbar_wait(&full[q % kFnoStages], (q / kFnoStages) & 1, kFnoWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(128, N);
      bool ok = mbar_wait(w_full, 0, kFnoWaitNs);
      if (!ok) fail(12);
      tc_fence_after();
      int it = 0;
      for (int t = blockIdx.x; t < p.tiles && ok && !*abort_flag; t += gridDim.x, ++it) {
        const int s = it % kFnoStages, buf = it & 1;
        if (!mbar_wait(&tempty[buf], ((it >> 1) & 1) ^ 1, kFnoWaitNs)) {
          fail(13);
          break;
        }
        if (!mbar_wait(&full[s], (it / kFnoStages) & 1, kFnoWaitNs)) {
          fail(14);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + buf * N;
        uint8_t* st = sS + s * kStage;
        const uint64_t av = smem_desc_sw128(smem_u32(st));
        const uint64_t bw = smem_desc_sw128(smem_u32(sW));
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) tc_mma_bf16(d, av + 2 * ks, bw + 2 * ks, idesc, ks > 0 ? 1u : 0u);
        if (MODE == 0) {
          const uint64_t at = smem_desc_sw128(smem_u32(st + kTile));
          const uint64_t bz = smem_desc_sw128(smem_u32(st + 2 * kTile));
          for (int ks = 0; ks < p.kk_steps; ++ks) tc_mma_bf16(d, at + 2 * ks, bz + 2 * ks, idesc, 1u);
        }
        tc_commit(&empty[s]);
        tc_commit(&tfull[buf]);
      }
      tc_commit(done);
      mbar_wait(done, 0, kFnoWaitNs);
    }
  } else {
    const int quad = warp & 3;
    const int row = quad * 32 + lane;
    int it = 0;
    for (int t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const int buf = it & 1;
      const bool got = __all_sync(0xffffffffu, mbar_wait(&tfull[buf], (it >> 1) & 1, kFnoWaitNs));
      if (!got) {
        if (lane == 0) fail(15);
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + buf * N;
      const size_t pix = static_cast<size_t>(t) * 128 + row;
      if (MODE == 0) {
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 32) {
          float v[32];
          tmem_ld32(taddr + c0, v);
          __align__(16) __nv_bfloat16 zb[32], vb[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float z = v[i] + __ldg(p.bias + c0 + i);
            zb[i] = __float2bfloat16_rn(z);
            vb[i] = __float2bfloat16_rn(p.act ? tc_gelu(z) : z);
          }
          uint4* zd = reinterpret_cast<uint4*>(p.zsave + pix * 64 + c0);
          uint4* vd = reinterpret_cast<uint4*>(p.vnext + pix * 64 + c0);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            zd[q] = reinterpret_cast<const uint4*>(zb)[q];
            vd[q] = reinterpret_cast<const uint4*>(vb)[q];
          }
        }
      } else {
        float acc = __ldg(p.b2);
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 32) {
          float v[32];
          tmem_ld32(taddr + c0, v);
#pragma unroll
          for (int i = 0; i < 32; ++i) acc += __ldg(p.q2 + c0 + i) * tc_gelu(v[i] + __ldg(p.bias + c0 + i));
        }
        p.out[pix] = acc;
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// ------------------------------------------------------------------ backward
// Backward of the pointwise layer on tcgen05, per 128-pixel tile:
//   dz = dvnext * GELU'(z)  (or dvnext for the last layer), stored (f32);
//   dv = dz W               (M 128 pixels, N 64 inputs, K 64 outputs), stored (f32);
//   dW += dz^T v, db += sum dz over the CTA's tiles.
// The elementwise part runs on CUDA cores (warps 5..20, two 8-channel chunks
// of 32 pixels per thread, coalesced 32-byte rows) and writes the operands of
// both GEMMs straight into shared memory in the 128B-swizzled K-major layout:
// sA[px][o] = dz (A of dv), sX[ch][px] = (dz^T; v^T) (A of dW, 128 rows x 128
// pixels in two 64-wide boxes; its rows 64..127, v^T, are also the B operand),
// sWT[i][o] = W[o][i] (B of dv, converted from the f32 weights once per CTA).
// dW is the top half of the 128 x 64 product (dz^T; v^T) v, accumulated in
// tensor memory over every tile of the CTA and added to global memory once;
// the bottom half (v^T v) is not used.  Warp 0 issues the MMAs (one thread),
// warps 1..4 drain dv from tensor memory (one lane quadrant each).  Operand
// stages and dv accumulators are double-buffered; one CTA per SM, persistent.
// Every mbarrier wait is bounded; a timeout sets *err and unwinds.
constexpr int kBwdXWarps = 16;                      // elementwise warps
constexpr int kBwdThreads = 32 * (5 + kBwdXWarps);  // MMA + 4 epilogue + elementwise
constexpr uint32_t kBwdStage = 16384 + 2 * 16384;   // sA + sX
constexpr size_t kBwdSmem = 1024 + 8192 + 2 * static_cast<size_t>(kBwdStage) + 256;

__device__ __forceinline__ float tc_gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// byte offset of element (row, k) in a K-major 128B-swizzled tile of 128-byte rows
__device__ __forceinline__ uint32_t sw128_off(int row, int k) {
  return static_cast<uint32_t>(row) * 128u + ((static_cast<uint32_t>(k >> 3) ^ static_cast<uint32_t>(row & 7)) << 4) +
         static_cast<uint32_t>(k & 7) * 2u;
}

struct FnoBwdParams {
  int tiles;
  int act;
  const float* dvnext;      // [pix][64]
  const __nv_bfloat16* z;   // [pix][64]
  const __nv_bfloat16* v;   // [pix][64]
  const float* W;           // [64 o][64 i]
  float* dz;                // [pix][64]
  float* dv;                // [pix][64]
  float* dW;                // [64][64], accumulated
  float* db;                // [64], accumulated
  int* err;
};

__global__ void __launch_bounds__(kBwdThreads, 1) fno_tc_layer_bwd(FnoBwdParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* sWT = base;               // [64 i][64 o]
  uint8_t* sS = base + 8192;         // [stage] { sA [128 px][64 o], sX [2 boxes][128 ch][64 px] }
  uint64_t* bars = reinterpret_cast<uint64_t*>(sS + 2 * kBwdStage);
  uint64_t* full = bars;             // [2], one arrival per elementwise warp
  uint64_t* empty = bars + 2;        // [2], MMA commit
  uint64_t* tfull = bars + 4;        // [2]
  uint64_t* tempty = bars + 6;       // [2], one arrival per epilogue warp
  uint64_t* done = bars + 8;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 9);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t kTmemCols = 256;  // dv accumulators at 0 / 64, dW at 128

  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&full[s], kBwdXWarps);
      mbar_init(&empty[s], 1);
      mbar_init(&tfull[s], 1);
      mbar_init(&tempty[s], 4);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  auto fail = [&](int code) {
    *abort_flag = 1;
    if (p.err) atomicExch(p.err, code);
  };

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(128, 64);
      const uint64_t bw = smem_desc_sw128(smem_u32(sWT));
      int it = 0;
      for (int t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x, ++it) {
        const int s = it & 1;
        if (!mbar_wait_or_abort(&tempty[s], ((it >> 1) & 1) ^ 1, kFnoWaitNs, abort_flag)) {
          fail(31);
          break;
        }
        if (!mbar_wait_or_abort(&full[s], (it >> 1) & 1, kFnoWaitNs, abort_flag)) {
          fail(32);
          break;
        }
        tc_fence_after();
        uint8_t* sA = sS + s * kBwdStage;
        uint8_t* sX = sA + 16384;
        const uint64_t aa = smem_desc_sw128(smem_u32(sA));
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) tc_mma_bf16(tmem_base + s * 64, aa + 2 * ks, bw + 2 * ks, idesc, ks > 0 ? 1u : 0u);
        tc_commit(&tfull[s]);
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          uint8_t* box = sX + (ks >> 2) * 16384;
          const uint64_t ax = smem_desc_sw128(smem_u32(box)) + 2 * (ks & 3);
          const uint64_t bx = smem_desc_sw128(smem_u32(box + 8192)) + 2 * (ks & 3);
          tc_mma_bf16(tmem_base + 128, ax, bx, idesc, (it > 0 || ks > 0) ? 1u : 0u);
        }
        tc_commit(&empty[s]);
      }
      tc_commit(done);
      mbar_wait(done, 0, kFnoWaitNs);
    }
  } else if (warp <= 4) {
    // dv epilogue: lane quadrant warp % 4, one pixel row per lane
    const int quad = warp & 3;
    int it = 0;
    for (int t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const int s = it & 1;
      const bool got =
          __all_sync(0xffffffffu, mbar_wait_or_abort(&tfull[s], (it >> 1) & 1, kFnoWaitNs, abort_flag));
      if (!got) {
        if (lane == 0) fail(33);
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + s * 64;
      float a[32], b[32];
      tmem_ld32(taddr, a);
      tmem_ld32(taddr + 32, b);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[s]);
      float4* o = reinterpret_cast<float4*>(p.dv + (static_cast<size_t>(t) * 128 + quad * 32 + lane) * 64);
#pragma unroll
      for (int q = 0; q < 8; ++q) o[q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
#pragma unroll
      for (int q = 0; q < 8; ++q) o[8 + q] = make_float4(b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
    }
    // dW rows o = lanes 0..63 of the second accumulator, once every MMA is complete
    if (quad < 2) {
      const bool fin = __all_sync(0xffffffffu, mbar_wait(done, 0, kFnoWaitNs));
      if (fin && !*abort_flag) {
        tc_fence_after();
        const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + 128;
        float a[32], b[32];
        tmem_ld32(taddr, a);
        tmem_ld32(taddr + 32, b);
        float* w = p.dW + (quad * 32 + lane) * 64;
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(w + i, a[i]);
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(w + 32 + i, b[i]);
      } else if (!fin && lane == 0) {
        fail(34);
      }
    }
  } else {
    // elementwise warps: channel group og (8 channels), pixels 32 (2 jb + c) + lane
    const int xw = warp - 5, og = xw & 7, jb = xw >> 3, o0 = 8 * og;
    const int xt = threadIdx.x - 5 * 32;
    // W^T into sWT once: element (o, i) of W is row i, column o of the B operand
    for (int e = xt; e < 64 * 64; e += 32 * kBwdXWarps) {
      const int o = e >> 6, i = e & 63;
      *reinterpret_cast<__nv_bfloat16*>(sWT + sw128_off(i, o)) = __float2bfloat16_rn(p.W[e]);
    }
    float dbp[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) dbp[e] = 0.f;
    int it = 0;
    for (int t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const int s = it & 1;
      float4 g[2][2];
      uint4 zz[2], vv[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int px = 32 * (2 * jb + c) + lane;
        const size_t off = (static_cast<size_t>(t) * 128 + px) * 64 + o0;
        g[c][0] = *reinterpret_cast<const float4*>(p.dvnext + off);
        g[c][1] = *reinterpret_cast<const float4*>(p.dvnext + off + 4);
        zz[c] = p.act ? *reinterpret_cast<const uint4*>(p.z + off) : make_uint4(0, 0, 0, 0);
        vv[c] = *reinterpret_cast<const uint4*>(p.v + off);
      }
      // stage s was last read by the MMAs of tile it - 2
      const bool ok = __all_sync(0xffffffffu, mbar_wait_or_abort(&empty[s], ((it >> 1) & 1) ^ 1, kFnoWaitNs, abort_flag));
      if (!ok) {
        if (lane == 0) fail(35);
        break;
      }
      uint8_t* sA = sS + s * kBwdStage;
      uint8_t* sX = sA + 16384;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int px = 32 * (2 * jb + c) + lane;
        const size_t off = (static_cast<size_t>(t) * 128 + px) * 64 + o0;
        const float gv[8] = {g[c][0].x, g[c][0].y, g[c][0].z, g[c][0].w, g[c][1].x, g[c][1].y, g[c][1].z, g[c][1].w};
        const __nv_bfloat16* zb = reinterpret_cast<const __nv_bfloat16*>(&zz[c]);
        const __nv_bfloat16* vb = reinterpret_cast<const __nv_bfloat16*>(&vv[c]);
        float d[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          d[e] = p.act ? gv[e] * tc_gelu_grad(__bfloat162float(zb[e])) : gv[e];
          dbp[e] += d[e];
        }
        reinterpret_cast<float4*>(p.dz + off)[0] = make_float4(d[0], d[1], d[2], d[3]);
        reinterpret_cast<float4*>(p.dz + off)[1] = make_float4(d[4], d[5], d[6], d[7]);
        __align__(16) __nv_bfloat16 db16[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) db16[e] = __float2bfloat16_rn(d[e]);
        // A of dv: row px, 16-byte chunk og
        *reinterpret_cast<uint4*>(sA + sw128_off(px, o0)) = *reinterpret_cast<const uint4*>(db16);
        // A of dW: rows o (dz^T) and 64 + i (v^T), column px
        uint8_t* box = sX + (px >> 6) * 16384;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          *reinterpret_cast<__nv_bfloat16*>(box + sw128_off(o0 + e, px & 63)) = db16[e];
          *reinterpret_cast<__nv_bfloat16*>(box + sw128_off(64 + o0 + e, px & 63)) = vb[e];
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
    }
    if (!*abort_flag) {
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        float x = dbp[e];
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) x += __shfl_xor_sync(0xffffffffu, x, sh);
        if (lane == 0) atomicAdd(p.db + o0 + e, x);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// Backward of the projection head on tcgen05, per 128-pixel tile (h = Q1 v + b1):
//   h - b1 = v Q1^T                 (M 128 px, N 128 j, K 64 c)   GEMM-h
//   dh = dout Q2 GELU'(h), g = dout GELU(h)                        CUDA cores
//   dv = dh Q1                      (M 128 px, N 64 c,  K 128 j)  GEMM-dv
//   [dQ1 | db1] += dh^T [v | 1]     (M 128 j,  N 80,    K 128 px) GEMM-Q
//   dQ2 += g^T 1                    (M 128 j,  N 16,    K 128 px) GEMM-G
//   db2 += sum dout.
// Warp 0 loads the v tile (TMA, 128B swizzle), warp 1 issues the MMAs (one
// thread), warps 2..9 (two per tensor-memory lane quadrant, each half of
// the columns) do the elementwise part, write the BF16 operands dh, dh^T,
// g^T and v^T into shared memory (128B-swizzled K-major), and drain dv.
// The weight-gradient sums stay in tensor memory over all tiles of the CTA
// and are added to global memory once.  One CTA per SM, persistent.
constexpr int kPbThreads = 320;
constexpr uint32_t kPbQ1 = 0, kPbQ1T = 16384, kPbOnes = 32768, kPbV = 36864, kPbDH = 53248, kPbDHT = 86016,
                   kPbGT = 118784, kPbBQ = 151552, kPbBars = 172032;
constexpr size_t kPbSmem = 1024 + kPbBars + 256;

struct FnoProjBwdParams {
  int tiles;
  const float* Q1;    // [128 j][64 c]
  const float* b1;    // [128]
  const float* q2;    // [128]
  const float* dout;  // [pix]
  float* dv;          // [pix][64]
  float* dQ1;         // [128][64], accumulated
  float* db1;         // [128]
  float* dQ2;         // [128]
  float* db2;         // [1]
  int* err;
};

__global__ void __launch_bounds__(kPbThreads, 1)
    fno_tc_proj_bwd(const __grid_constant__ CUtensorMap tmV, FnoProjBwdParams p) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kPbBars);
  uint64_t* v_full = bars + 0;
  uint64_t* v_free = bars + 1;   // GEMM-h commit + 8 elementwise warps
  uint64_t* h_full = bars + 2;
  uint64_t* h_free = bars + 3;   // 8 elementwise warps
  uint64_t* ops_full = bars + 4; // 8 elementwise warps
  uint64_t* ops_free = bars + 5;
  uint64_t* dv_full = bars + 6;
  uint64_t* dv_free = bars + 7;  // 8 elementwise warps
  uint64_t* w_ready = bars + 8;  // 8 elementwise warps
  uint64_t* done = bars + 9;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 10);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t kTmemCols = 512;
  constexpr uint32_t cH = 0, cDV = 128, cQ = 192, cG = 272;  // accumulator columns

  if (threadIdx.x == 0) {
    mbar_init(v_full, 1);
    mbar_init(v_free, 9);
    mbar_init(h_full, 1);
    mbar_init(h_free, 8);
    mbar_init(ops_full, 8);
    mbar_init(ops_free, 1);
    mbar_init(dv_full, 1);
    mbar_init(dv_free, 8);
    mbar_init(w_ready, 8);
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  auto fail = [&](int code) {
    *abort_flag = 1;
    if (p.err) atomicExch(p.err, code);
  };

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&tmV);
      int it = 0;
      for (int t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x, ++it) {
        if (!mbar_wait_or_abort(v_free, (it & 1) ^ 1, kFnoWaitNs, abort_flag)) {
          fail(41);
          break;
        }
        mbar_arrive_expect_tx(v_full, kTile);
        tma_load_2d(base + kPbV, &tmV, 0, t * 128, v_full);
      }
      // the last load issued lands before the CTA may exit
      if (it > 0) mbar_wait(v_full, (it - 1) & 1, kFnoWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = mbar_wait_or_abort(w_ready, 0, kFnoWaitNs, abort_flag);
      if (!ok) fail(42);
      int it = 0;
      for (int t = blockIdx.x; t < p.tiles && ok && !*abort_flag; t += gridDim.x, ++it) {
        const uint32_t ph = it & 1;
        if (!mbar_wait_or_abort(v_full, ph, kFnoWaitNs, abort_flag) ||
            !mbar_wait_or_abort(h_free, ph ^ 1, kFnoWaitNs, abort_flag)) {
          fail(43);
          break;
        }
        tc_fence_after();
        {
          const uint64_t a = smem_desc_sw128(smem_u32(base + kPbV));
          const uint64_t b = smem_desc_sw128(smem_u32(base + kPbQ1));
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            tc_mma_bf16(tmem_base + cH, a + 2 * ks, b + 2 * ks, idesc_bf16(128, 128), ks > 0 ? 1u : 0u);
        }
        tc_commit(h_full);
        tc_commit(v_free);
        if (!mbar_wait_or_abort(ops_full, ph, kFnoWaitNs, abort_flag) ||
            !mbar_wait_or_abort(dv_free, ph ^ 1, kFnoWaitNs, abort_flag)) {
          fail(44);
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          const uint32_t bx = ks >> 2, kk = 2 * (ks & 3);
          tc_mma_bf16(tmem_base + cDV, smem_desc_sw128(smem_u32(base + kPbDH + bx * 16384)) + kk,
                      smem_desc_sw128(smem_u32(base + kPbQ1T + bx * 8192)) + kk, idesc_bf16(128, 64),
                      ks > 0 ? 1u : 0u);
        }
        tc_commit(dv_full);
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          const uint32_t bx = ks >> 2, kk = 2 * (ks & 3);
          const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
          tc_mma_bf16(tmem_base + cQ, smem_desc_sw128(smem_u32(base + kPbDHT + bx * 16384)) + kk,
                      smem_desc_sw128(smem_u32(base + kPbBQ + bx * 10240)) + kk, idesc_bf16(128, 80), acc);
          tc_mma_bf16(tmem_base + cG, smem_desc_sw128(smem_u32(base + kPbGT + bx * 16384)) + kk,
                      smem_desc_sw128(smem_u32(base + kPbOnes + bx * 2048)) + kk, idesc_bf16(128, 16), acc);
        }
        tc_commit(ops_free);
      }
      tc_commit(done);
      mbar_wait(done, 0, kFnoWaitNs);
    }
  } else {
    // elementwise warps 2..9: lane quadrant warp % 4 (pixel rows of a tile,
    // j rows of the weight-gradient sums), column half `half`
    const int quad = warp & 3, half = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;  // 0..255
    // resident operands: Q1 [j][c] (B of GEMM-h), Q1^T [c][j] (B of GEMM-dv),
    // ones (B of GEMM-G: row 0), rows 64..79 of [v^T; 1] (row 64 ones)
    for (int e = et; e < 128 * 64; e += 256) {
      const int j = e >> 6, c = e & 63;
      const __nv_bfloat16 q = __float2bfloat16_rn(p.Q1[e]);
      *reinterpret_cast<__nv_bfloat16*>(base + kPbQ1 + sw128_off(j, c)) = q;
      *reinterpret_cast<__nv_bfloat16*>(base + kPbQ1T + (j >> 6) * 8192 + sw128_off(c, j & 63)) = q;
    }
    const __nv_bfloat16 one = __float2bfloat16_rn(1.f), zero = __float2bfloat16_rn(0.f);
    for (int e = et; e < 2 * 16 * 64; e += 256) {
      const int bx = e >> 10, r = (e >> 6) & 15, k = e & 63;
      *reinterpret_cast<__nv_bfloat16*>(base + kPbOnes + bx * 2048 + sw128_off(r, k)) = r == 0 ? one : zero;
      *reinterpret_cast<__nv_bfloat16*>(base + kPbBQ + bx * 10240 + sw128_off(64 + r, k)) = r == 0 ? one : zero;
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive(w_ready);

    const int px = quad * 32 + lane;  // pixel row within the tile
    const int bxp = px >> 6, kp = px & 63;
    float gd2 = 0.f;
    int it = 0;
    for (int t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const uint32_t ph = it & 1;
      const bool ok = __all_sync(0xffffffffu, mbar_wait_or_abort(h_full, ph, kFnoWaitNs, abort_flag) &&
                                                  mbar_wait_or_abort(ops_free, ph ^ 1, kFnoWaitNs, abort_flag));
      if (!ok) {
        if (lane == 0) fail(45);
        break;
      }
      tc_fence_after();
      const float d = p.dout[static_cast<size_t>(t) * 128 + px];
      if (half == 0) gd2 += d;
#pragma unroll 1
      for (int jc = 0; jc < 2; ++jc) {
        const int j0 = half * 64 + jc * 32;
        float h[32];
        tmem_ld32(tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + cH + j0, h);
        __align__(16) __nv_bfloat16 dhb[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int j = j0 + i;
          const float x = h[i] + __ldg(p.b1 + j);
          const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
          const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
          const float dh = d * __ldg(p.q2 + j) * (cdf + x * pdf);
          dhb[i] = __float2bfloat16_rn(dh);
          const __nv_bfloat16 gb = __float2bfloat16_rn(d * x * cdf);
          // dh^T and g^T: row j, column px (2-byte stores, one row per warp store)
          *reinterpret_cast<__nv_bfloat16*>(base + kPbDHT + bxp * 16384 + sw128_off(j, kp)) = dhb[i];
          *reinterpret_cast<__nv_bfloat16*>(base + kPbGT + bxp * 16384 + sw128_off(j, kp)) = gb;
        }
        // dh: row px, four 16-byte chunks of 8 j
        uint8_t* dbox = base + kPbDH + (j0 >> 6) * 16384;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4*>(dbox + sw128_off(px, (j0 & 63) + 8 * q)) = reinterpret_cast<const uint4*>(dhb)[q];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(h_free);
      // v^T rows c (this half's 32 channels), column px, from the v tile
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c0 = half * 32 + 8 * q;
        const uint4 w = *reinterpret_cast<const uint4*>(base + kPbV + sw128_off(px, c0));
        const __nv_bfloat16* vb = reinterpret_cast<const __nv_bfloat16*>(&w);
#pragma unroll
        for (int e = 0; e < 8; ++e)
          *reinterpret_cast<__nv_bfloat16*>(base + kPbBQ + bxp * 10240 + sw128_off(c0 + e, kp)) = vb[e];
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(v_free);
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(ops_full);
      // dv: this half's 32 channels of pixel row px
      const bool got = __all_sync(0xffffffffu, mbar_wait_or_abort(dv_full, ph, kFnoWaitNs, abort_flag));
      if (!got) {
        if (lane == 0) fail(46);
        break;
      }
      tc_fence_after();
      float o[32];
      tmem_ld32(tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + cDV + half * 32, o);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(dv_free);
      float4* dst = reinterpret_cast<float4*>(p.dv + (static_cast<size_t>(t) * 128 + px) * 64 + half * 32);
#pragma unroll
      for (int q = 0; q < 8; ++q) dst[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
    }
    // weight-gradient sums: rows j = lanes of the quadrant
    const bool fin = __all_sync(0xffffffffu, mbar_wait(done, 0, kFnoWaitNs));
    if (fin && !*abort_flag) {
      tc_fence_after();
      const int j = quad * 32 + lane;
      const uint32_t lrow = static_cast<uint32_t>(quad * 32) << 16;
      float a[32];
      tmem_ld32(tmem_base + lrow + cQ + half * 32, a);
#pragma unroll
      for (int i = 0; i < 32; ++i) atomicAdd(p.dQ1 + j * 64 + half * 32 + i, a[i]);
      if (half == 0) {
        float b[16], g[16];
        tmem_ld16(tmem_base + lrow + cQ + 64, b);
        tmem_ld16(tmem_base + lrow + cG, g);
        atomicAdd(p.db1 + j, b[0]);
        atomicAdd(p.dQ2 + j, g[0]);
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) gd2 += __shfl_xor_sync(0xffffffffu, gd2, sh);
        if (lane == 0) atomicAdd(p.db2, gd2);
      }
    } else if (!fin && lane == 0) {
      fail(47);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// bf16 copy of an fp32 matrix (weights for the tensor-core operands).
__global__ void fno_to_bf16(const float* __restrict__ a, int n, __nv_bfloat16* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn(a[i]);
}

// Zs[r][o][kk] (bf16, kk < 64): kk = 2 kx -> w Re Z, 2 kx + 1 -> -w Im Z,
// w = (kx ? 2 : 1) / S^2, zero for kk >= 2m; Z: [r][kx][o] float2 (r = b S + y).
__global__ void fno_zs_pack(const float2* __restrict__ Z, int rows, int m, int S, __nv_bfloat16* __restrict__ Zs) {
  const float inv = 1.f / (static_cast<float>(S) * S);
  const size_t total = static_cast<size_t>(rows) * 64 * 64;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int kk = static_cast<int>(t & 63), o = static_cast<int>((t >> 6) & 63);
    const size_t r = t >> 12;
    float v = 0.f;
    if (kk < 2 * m) {
      const int kx = kk >> 1;
      const float w = (kx == 0 ? 1.f : 2.f) * inv;
      const float2 z = Z[(r * m + kx) * 64 + o];
      v = (kk & 1) ? -w * z.y : w * z.x;
    }
    Zs[t] = __float2bfloat16_rn(v);
  }
}

// Tw[x][kk] (bf16): cos / sin of 2 pi kx x / S for kk = 2 kx / 2 kx + 1 < 2m,
// zero beyond; from twx[kx][x] = (cos, -sin).
__global__ void fno_tw_table(const float2* __restrict__ twx, int S, int m, __nv_bfloat16* __restrict__ Tw) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < S * 64; t += gridDim.x * blockDim.x) {
    const int kk = t & 63, x = t >> 6;
    float v = 0.f;
    if (kk < 2 * m) {
      const float2 w = twx[static_cast<size_t>(kk >> 1) * S + x];
      v = (kk & 1) ? -w.y : w.x;
    }
    Tw[t] = __float2bfloat16_rn(v);
  }
}

}  // namespace huv_dev

namespace huv_launch {
bool tc_map_bf16(CUtensorMap* map, const void* ptr, uint64_t rows, int kp, int box_rows);

size_t fno_tc_smem(int mode) {
  const size_t w = (mode == 0 ? 64 : 128) * 128;
  const size_t stage = mode == 0 ? 2 * huv_dev::kTile + 64 * 128 : huv_dev::kTile;
  return 1024 + w + huv_dev::kFnoStages * stage + 256;
}

cudaError_t fno_tc_set_smem() {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(huv_dev::fno_tc_pw<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(fno_tc_smem(0)))))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::fno_tc_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(huv_dev::kBwdSmem))))
    return e;
  if ((e = cudaFuncSetAttribute(huv_dev::fno_tc_proj_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(huv_dev::kPbSmem))))
    return e;
  return cudaFuncSetAttribute(huv_dev::fno_tc_pw<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(fno_tc_smem(1)));
}

// Layer l forward on tensor cores.  v: [B*S*S][64] bf16; Wb: [64][64] bf16;
// Tw: [S][64] bf16; Zs: [B*S*64][64] bf16.
bool fno_tc_layer(int B, int S, int m, const __nv_bfloat16* v, const __nv_bfloat16* Wb,
                  const __nv_bfloat16* Tw, const __nv_bfloat16* Zs, const float* bias, int act,
                  __nv_bfloat16* zsave, __nv_bfloat16* vnext, int* err, cudaStream_t st) {
  CUtensorMap mv, mw, mt, mz;
  const uint64_t pix = static_cast<uint64_t>(B) * S * S;
  if (!tc_map_bf16(&mv, v, pix, 64, 128) || !tc_map_bf16(&mw, Wb, 64, 64, 64) ||
      !tc_map_bf16(&mt, Tw, static_cast<uint64_t>(S), 64, 128) ||
      !tc_map_bf16(&mz, Zs, static_cast<uint64_t>(B) * S * 64, 64, 64))
    return false;
  huv_dev::FnoTcParams p{};
  p.tiles = static_cast<int>(pix / 128);
  p.S = S;
  p.kk_steps = (2 * m + 15) / 16;
  p.bias = bias;
  p.zsave = zsave;
  p.vnext = vnext;
  p.act = act;
  p.err = err;
  const int grid = std::min(p.tiles, 2 * 148);
  huv_dev::fno_tc_pw<0><<<grid, 192, fno_tc_smem(0), st>>>(mv, mw, mt, mz, p);
  return cudaGetLastError() == cudaSuccess;
}

// Projection head on tensor cores.  Q1b: [128][64] bf16.
bool fno_tc_proj(int B, int S, const __nv_bfloat16* v, const __nv_bfloat16* Q1b, const float* b1, const float* q2,
                 const float* b2, float* out, int* err, cudaStream_t st) {
  CUtensorMap mv, mq;
  const uint64_t pix = static_cast<uint64_t>(B) * S * S;
  if (!tc_map_bf16(&mv, v, pix, 64, 128) || !tc_map_bf16(&mq, Q1b, 128, 64, 128)) return false;
  huv_dev::FnoTcParams p{};
  p.tiles = static_cast<int>(pix / 128);
  p.S = S;
  p.bias = b1;
  p.q2 = q2;
  p.b2 = b2;
  p.out = out;
  p.err = err;
  const int grid = std::min(p.tiles, 2 * 148);
  huv_dev::fno_tc_pw<1><<<grid, 192, fno_tc_smem(1), st>>>(mv, mq, mq, mq, p);
  return cudaGetLastError() == cudaSuccess;
}
// Layer backward on tensor cores (see fno_tc_layer_bwd); pix a multiple of 128.
bool fno_tc_layer_bwd(size_t pix, const float* dvnext, const __nv_bfloat16* z, const __nv_bfloat16* v, const float* W,
                      int act, float* dz, float* dv, float* dW, float* db, int* err, cudaStream_t st) {
  if (pix % 128 != 0) return false;
  huv_dev::FnoBwdParams p{};
  p.tiles = static_cast<int>(pix / 128);
  p.act = act;
  p.dvnext = dvnext;
  p.z = z;
  p.v = v;
  p.W = W;
  p.dz = dz;
  p.dv = dv;
  p.dW = dW;
  p.db = db;
  p.err = err;
  int sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  const int grid = std::min(p.tiles, sms);
  huv_dev::fno_tc_layer_bwd<<<grid, huv_dev::kBwdThreads, huv_dev::kBwdSmem, st>>>(p);
  return cudaGetLastError() == cudaSuccess;
}
// Projection backward on tensor cores (see fno_tc_proj_bwd); v: [pix][64]
// bf16, pix a multiple of 128.
bool fno_tc_proj_bwd(size_t pix, const __nv_bfloat16* v, const float* Q1, const float* b1, const float* q2,
                     const float* dout, float* dv, float* dQ1, float* db1, float* dQ2, float* db2, int* err,
                     cudaStream_t st) {
  if (pix % 128 != 0) return false;
  CUtensorMap mv;
  if (!tc_map_bf16(&mv, v, pix, 64, 128)) return false;
  huv_dev::FnoProjBwdParams p{};
  p.tiles = static_cast<int>(pix / 128);
  p.Q1 = Q1;
  p.b1 = b1;
  p.q2 = q2;
  p.dout = dout;
  p.dv = dv;
  p.dQ1 = dQ1;
  p.db1 = db1;
  p.dQ2 = dQ2;
  p.db2 = db2;
  p.err = err;
  int sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  const int grid = std::min(p.tiles, sms);
  huv_dev::fno_tc_proj_bwd<<<grid, huv_dev::kPbThreads, huv_dev::kPbSmem, st>>>(mv, p);
  return cudaGetLastError() == cudaSuccess;
}
void fno_tc_to_bf16(const float* a, int n, __nv_bfloat16* b, cudaStream_t st) {
  huv_dev::fno_to_bf16<<<(n + 255) / 256, 256, 0, st>>>(a, n, b);
}
void fno_tc_pack_zs(const float2* Z, int rows, int m, int S, __nv_bfloat16* Zs, cudaStream_t st) {
  huv_dev::fno_zs_pack<<<2048, 256, 0, st>>>(Z, rows, m, S, Zs);
}
void fno_tc_tw_table(const float2* twx, int S, int m, __nv_bfloat16* Tw, cudaStream_t st) {
  huv_dev::fno_tw_table<<<(S * 64 + 255) / 256, 256, 0, st>>>(twx, S, m, Tw);
}
}  // namespace huv_launch
