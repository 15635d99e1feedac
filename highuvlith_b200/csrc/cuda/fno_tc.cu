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
