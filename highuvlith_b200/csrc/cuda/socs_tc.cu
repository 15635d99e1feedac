// Tensor-core (split-BF16x3, tcgen05) form of the SOCS aerial image, sm_100a.
//
// The cropped-band inverse transform along y is a dense DFT-matrix
// contraction.  For every kernel k the per-kernel field on the evaluation
// grid is E_k(y, x) = sum_my G(y, my) T_k(my, x), with T_k the row transform
// (FFT along x, FP32) of the band product K_k . M.  Complex arithmetic is laid
// out as a real GEMM whose rows are (y, re/im) pairs:
//     row (y, re) = [ cos t, -sin t ] , row (y, im) = [ sin t, cos t ]
// against B rows x = [ Tr(my), Ti(my) ] (K index 2 my + re/im).  Each FP32
// value v is split v = hi + lo (two BF16 planes) and the product is taken as
// hi.hi + hi.lo + lo.hi with FP32 accumulation in tensor memory; B's hi plane
// is read twice from the same shared-memory tile.  The epilogue squares the
// accumulator, combines the (re, im) lanes with one shuffle and sums
// lambda_k |E_k|^2 over k in registers (lambda folded into the kernels), then
// applies normalisation and flare.  The same kernel, in store mode, performs
// the exact band interpolation from the evaluation grid to the N x N output
// (Hermitian half band, real part only).
//
// Roles per CTA (6 warps): warp 0 issues TMA loads (no multicast), warp 1
// issues tcgen05.mma from one thread, warps 2-5 drain tensor memory.  All
// mbarrier waits are bounded in time; a timeout sets an error flag, drains
// in-flight work with bounded waits, frees tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "../engine.hpp"
#include "fft_block.cuh"
#include "fft_reg.cuh"
#include "tc_ptx.cuh"

namespace huv_dev {

constexpr int kTcStages = 3;
constexpr int kTcBN = 128;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s per wait
constexpr uint32_t kABox = 128 * 128;             // 128 rows x 64 bf16
// B box of BN rows x 64 bf16
__host__ __device__ constexpr uint32_t b_box_bytes(int bn) { return static_cast<uint32_t>(bn) * 128; }
// Row-transform GEMM (MODE 2): N = band rows padded to 80 (B <= 80) or 96
// (B <= 96, the largest band whose operand rows fit K = 192).
constexpr int kRowBN = 80;
constexpr int kRowBNWide = 96;
// per epilogue warp: [plane][16 x][BN (+1 pad) my] bf16x2
__host__ __device__ constexpr int stage_words(int bn) { return 2 * 16 * (bn + 1); }

struct TcGemmParams {
  int kboxes;       // 64-wide K boxes loaded
  int ksteps;       // 16-wide MMA K steps issued
  int G;            // steps per CTA: kernels (MODE 0) or x tiles (MODE 1)
  int a_rows;       // rows of A per split plane
  int b_prob;       // B rows between problems
  int b_step;       // B rows between steps
  int b_plane;      // B rows between the hi and lo planes
  int out_ld;       // output row stride (floats)
  long long out_plane;
  float keep, flare;
  const float* mean;
  float* out;
  int* err;
  // MODE 2 output: split-BF16 operand rows, Bop[g][plane][x][2 my + re/im]
  __nv_bfloat16* bop;
  long long bop_g;      // elements between steps (kernels)
  long long bop_prob;   // elements between problems
  long long bop_plane;  // elements between the hi and lo planes
  int bop_ld;           // row stride (elements)
  int bop_cols;         // band rows my written (2 bop_cols <= bop_ld)
  // MODE 1: 1 = store the output tiles with TMA (tmO) through shared memory
  int out_tma;
  // MODE 3: problems in all; CTA z takes problems z G .. z G + G - 1
  int nprob;
  // A and B are FP16 planes (else BF16); MODE 3 always
  int f16;
  // > 0: before its first MMA the MMA-issuing thread waits this long on a
  // barrier nothing arrives at, so the wait runs out and the kernel takes
  // its give-up path (a test of the bounded waits; 0 in normal use)
  unsigned long long probe_wait_ns;
};

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// MODE 1 output staging: per epilogue warp two 32 x 32 f32 tiles (128B swizzle).
constexpr uint32_t kOutTile = 32 * 32 * 4;
constexpr uint32_t kOutStage = 4 * 2 * kOutTile;

// B stages of the ring: MODE 3 fills 120 KB with as many as fit (3 to 8:
// its CTAs are bound by how much of B is in flight), the others take 3.
__host__ __device__ constexpr int tc_stages(int mode, int bn) {
  return mode != 3 ? kTcStages
                   : (122880 / (2 * static_cast<int>(b_box_bytes(bn))) > 8
                          ? 8
                          : (122880 / (2 * static_cast<int>(b_box_bytes(bn))) < kTcStages
                                 ? kTcStages
                                 : 122880 / (2 * static_cast<int>(b_box_bytes(bn)))));
}

__host__ __device__ constexpr size_t tc_smem_bytes(int kboxes, int bn = kTcBN, bool stage = false,
                                                   bool out_stage = false, int stages = kTcStages) {
  return 1024 + 2 * static_cast<size_t>(kboxes) * kABox + stages * 2 * static_cast<size_t>(b_box_bytes(bn)) +
         (out_stage ? kOutStage : 0) + 256 + (stage ? 4 * static_cast<size_t>(stage_words(bn)) * sizeof(uint32_t) : 0);
}

// MODE 0: sum over G steps (kernels) of |E|^2 with (re, im) in adjacent
// accumulator rows; out(y, x) = keep * sum + flare * mean[problem];
// grid: (x tiles, a_rows / 128, problems).  MODE 1: step g is x tile g of the
// same rows (the A tile stays resident), out(y, g * BN + j) = accumulator;
// grid: (1, a_rows / 128, problems).  MODE 2: step g is kernel g; the
// accumulator rows are (x, re/im), its columns band rows my; the tile is
// split into BF16 hi/lo and written, through shared memory, as rows x of the
// next GEMM's operand: bop[g][plane][x][2 my + re/im]; grid as MODE 1.
// MODE 1 with p.out_tma: each epilogue warp stages 32 x 32 tiles in shared
// memory (128B swizzle, double-buffered) and stores them with TMA through
// tmO, a [problems * a_rows][out_ld] f32 map with 32 x 32 boxes; MODE 1 with
// p.mean multiplies the tile by interp_scale(mean[problem]).  MODE 3: step g
// is problem z G + g (the A tile stays resident across problems); the
// accumulator tile (rows of A, columns n_tile BN + j) is split into FP16
// hi/lo and stored row by row as bop[problem][plane][row][col] (half
// elements); grid: (column tiles, a_rows / 128, ceil(nprob / G)).
template <int MODE, int BN = kTcBN>
__global__ void __launch_bounds__(192, 1)
    tc_dft_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmO, TcGemmParams p) {
  constexpr uint32_t kBBox = b_box_bytes(BN);
  constexpr uint32_t kTmemCols = 2 * BN <= 128 ? 128 : (2 * BN <= 256 ? 256 : 512);
  constexpr int kSt = tc_stages(MODE, BN);
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* sA = base;
  uint8_t* sB = base + 2 * p.kboxes * kABox;
  uint8_t* sO = sB + kSt * 2 * kBBox;  // MODE 1 output staging (1024-aligned)
  uint64_t* bars = reinterpret_cast<uint64_t*>(sO + (MODE == 1 ? kOutStage : 0));
  uint64_t* full = bars;
  uint64_t* empty = bars + kSt;
  uint64_t* a_full = bars + 2 * kSt;
  uint64_t* tfull = bars + 2 * kSt + 1;
  uint64_t* tempty = bars + 2 * kSt + 3;
  uint64_t* done = bars + 2 * kSt + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kSt + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_tile = blockIdx.x, m_tile = blockIdx.y, prob = blockIdx.z;
  // steps of this CTA (MODE 3: the last group of problems may be short)
  const int G = MODE == 3 ? min(p.G, p.nprob - prob * p.G) : p.G;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kSt; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(a_full, 1);
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

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&tmA);
      prefetch_tmap(&tmB);
      mbar_arrive_expect_tx(a_full, 2u * p.kboxes * kABox);
      for (int part = 0; part < 2; ++part)
        for (int kb = 0; kb < p.kboxes; ++kb)
          tma_load_2d(sA + (part * p.kboxes + kb) * kABox, &tmA, kb * 64, part * p.a_rows + m_tile * 128, a_full);
      int it = 0;
      for (int g = 0; g < G && !*abort_flag; ++g) {
        for (int kb = 0; kb < p.kboxes; ++kb, ++it) {
          const int s = it % kSt;
          const uint32_t ph = (it / kSt) & 1;
          if (!mbar_wait_or_abort(&empty[s], ph ^ 1, kWaitLimitNs, abort_flag)) {
            fail(1);
            break;
          }
          mbar_arrive_expect_tx(&full[s], 2u * kBBox);
          const int row = prob * p.b_prob + g * p.b_step + n_tile * BN;
          tma_load_2d(sB + (s * 2 + 0) * kBBox, &tmB, kb * 64, row, &full[s]);
          tma_load_2d(sB + (s * 2 + 1) * kBBox, &tmB, kb * 64, row + p.b_plane, &full[s]);
        }
      }
      // Drain: every load issued must have landed before the CTA may exit.
      mbar_wait(a_full, 0, kWaitLimitNs);
      for (int q = (it > kSt ? it - kSt : 0); q < it; ++q)
        mbar_wait(&full[q % kSt], (q / kSt) & 1, kWaitLimitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = (MODE == 3 || p.f16) ? idesc_f16(128, BN) : idesc_bf16(128, BN);
      bool ok = mbar_wait(a_full, 0, kWaitLimitNs);
      if (!ok) fail(2);
      if (ok && p.probe_wait_ns && !mbar_wait(done, 0, p.probe_wait_ns)) {  // nothing arrives at `done` yet
        fail(6);
        ok = false;
      }
      tc_fence_after();
      int it = 0;
      for (int g = 0; g < G && ok && !*abort_flag; ++g) {
        const int buf = g & 1;
        if (!mbar_wait_or_abort(&tempty[buf], ((g >> 1) & 1) ^ 1, kWaitLimitNs, abort_flag)) {
          fail(3);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + buf * BN;
        for (int kb = 0; kb < p.kboxes; ++kb, ++it) {
          const int s = it % kSt;
          if (!mbar_wait(&full[s], (it / kSt) & 1, kWaitLimitNs)) {
            fail(4);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t a_hi = smem_desc_sw128(smem_u32(sA + (0 * p.kboxes + kb) * kABox));
          const uint64_t a_lo = smem_desc_sw128(smem_u32(sA + (1 * p.kboxes + kb) * kABox));
          const uint64_t b_hi = smem_desc_sw128(smem_u32(sB + (s * 2 + 0) * kBBox));
          const uint64_t b_lo = smem_desc_sw128(smem_u32(sB + (s * 2 + 1) * kBBox));
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const int kstep = kb * 4 + ks;
            if (kstep < p.ksteps) {
              const uint64_t adv = static_cast<uint64_t>(2 * ks);  // 32 bytes per 16-wide K step
              tc_mma_bf16(d, a_hi + adv, b_hi + adv, idesc, kstep > 0 ? 1u : 0u);
              tc_mma_bf16(d, a_hi + adv, b_lo + adv, idesc, 1u);
              tc_mma_bf16(d, a_lo + adv, b_hi + adv, idesc, 1u);
            }
          }
          tc_commit(&empty[s]);
        }
        if (!ok) break;
        tc_commit(&tfull[buf]);
      }
      // All MMAs issued by this thread have completed once `done` flips.
      tc_commit(done);
      mbar_wait(done, 0, kWaitLimitNs);
    }
  } else {
    // Epilogue warps 2..5: TMEM lane quadrant = warp % 4.
    const int quad = warp & 3;
    const int row = quad * 32 + lane;  // accumulator row within the tile
    constexpr int HALF = BN / 2;
    // MODE 2 staging: after the 256 bytes of barriers, kStageWords per warp
    constexpr int SLD = BN + 1;  // staging row stride (words)
    uint32_t* stage = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(bars) + 256) + quad * stage_words(BN);
    float acc[MODE == 0 ? HALF : 1];
#pragma unroll
    for (int i = 0; i < (MODE == 0 ? HALF : 1); ++i) acc[i] = 0.f;
    const int odd = lane & 1;
    bool ok = true;
    int nst = 0;  // MODE 1 TMA-store tiles issued by this warp
    const float osc = (MODE == 1 && p.mean) ? interp_scale(p.mean[prob]) : 1.f;
    for (int g = 0; g < G; ++g) {
      const int buf = g & 1;
      // Warp-uniform outcome: tcgen05.ld below is .sync.aligned.
      const bool got = __all_sync(0xffffffffu, mbar_wait_or_abort(&tfull[buf], (g >> 1) & 1, kWaitLimitNs, abort_flag));
      if (!got) {
        if (lane == 0) fail(5);
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + buf * BN;
      if (MODE == 2) {
        // rows (x, re/im) in adjacent lanes: even lanes keep the hi pair of
        // (re, im), odd lanes the lo pair; staged as [plane][x][my].
        const int xl = lane >> 1;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          float v[16];
          tmem_ld16(taddr + c0, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float other = __shfl_xor_sync(0xffffffffu, v[i], 1);
            const float re = odd ? other : v[i], im = odd ? v[i] : other;
            __nv_bfloat16 rh, rl, ih, il;
            split_bf16(re, rh, rl);
            split_bf16(im, ih, il);
            __nv_bfloat162 pr;
            pr.x = odd ? rl : rh;
            pr.y = odd ? il : ih;
            stage[(odd * 16 + xl) * SLD + c0 + i] = *reinterpret_cast<uint32_t*>(&pr);
          }
        }
        __syncwarp();
        // coalesced copy-out: 32 rows (2 planes x 16 x) of bop_cols bf16 pairs
        const int x0 = (m_tile * 128 + quad * 32) >> 1;
        const int nc = p.bop_cols;
        uint32_t* base_out = reinterpret_cast<uint32_t*>(p.bop + prob * p.bop_prob + g * p.bop_g);
        for (int w = lane; w < 32 * nc; w += 32) {
          const int r = w / nc, my = w - r * nc;
          const int pl = r >> 4, x = x0 + (r & 15);
          base_out[(pl * p.bop_plane + static_cast<long long>(x) * p.bop_ld) / 2 + my] = stage[r * SLD + my];
        }
        __syncwarp();
      }
      if (MODE == 3) {
        // one accumulator row per lane: row X of problem prob G + g
        const long long X = m_tile * 128 + row;
        __half* hi = reinterpret_cast<__half*>(p.bop) + (static_cast<long long>(prob) * p.G + g) * p.bop_prob +
                     X * p.bop_ld + n_tile * BN;
        __half* lo = hi + p.bop_plane;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          float v[16];
          tmem_ld16(taddr + c0, v);
          uint32_t hw[8], lw[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const __half2 h2 = __floats2half2_rn(v[2 * i], v[2 * i + 1]);
            const float2 hf = __half22float2(h2);
            const __half2 l2 = __floats2half2_rn(v[2 * i] - hf.x, v[2 * i + 1] - hf.y);
            hw[i] = *reinterpret_cast<const uint32_t*>(&h2);
            lw[i] = *reinterpret_cast<const uint32_t*>(&l2);
          }
          uint4* hq = reinterpret_cast<uint4*>(hi + c0);
          uint4* lq = reinterpret_cast<uint4*>(lo + c0);
          hq[0] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
          hq[1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
          lq[0] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
          lq[1] = make_uint4(lw[4], lw[5], lw[6], lw[7]);
        }
      }
#pragma unroll
      for (int c0 = 0; c0 < (MODE >= 2 ? 0 : BN); c0 += 32) {
        float v[32];
        tmem_ld32(taddr + c0, v);
        if (MODE == 1 && p.mean) {
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] *= osc;
        }
        if (MODE == 0) {
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            float e = v[i] * v[i];
            e += __shfl_xor_sync(0xffffffffu, e, 1);
            const int j = c0 + i;
            if ((j / HALF) == odd) acc[j % HALF] += e;
          }
        } else if (p.out_tma) {
          // buffer `sb` was last read by the store issued two tiles ago
          const int sbuf = nst & 1;
          if (lane == 0 && nst >= 2) bulk_wait_read<1>();
          __syncwarp();
          uint8_t* sb = sO + (quad * 2 + sbuf) * kOutTile;
#pragma unroll
          for (int q = 0; q < 8; ++q)
            *reinterpret_cast<float4*>(sb + lane * 128 + ((q ^ (lane & 7)) << 4)) =
                make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(&tmO, sb, g * BN + c0, prob * p.a_rows + m_tile * 128 + quad * 32);
            bulk_commit();
          }
          ++nst;
        } else {
          const int y = m_tile * 128 + row;
          float* o = p.out + prob * p.out_plane + static_cast<long long>(y) * p.out_ld + g * BN + c0;
#pragma unroll
          for (int i = 0; i < 32; i += 4)
            *reinterpret_cast<float4*>(o + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
    // Every TMA store must have finished before the CTA's shared memory goes.
    if (MODE == 1 && lane == 0 && nst > 0) bulk_wait<0>();
    __syncwarp();
    if (MODE == 0 && ok) {
      const int y = (m_tile * 128 + row) >> 1;
      const float add = p.mean ? p.flare * p.mean[prob] : 0.f;
      float* o = p.out + prob * p.out_plane + static_cast<long long>(y) * p.out_ld + n_tile * BN + odd * HALF;
#pragma unroll
      for (int i = 0; i < HALF; i += 4)
        *reinterpret_cast<float4*>(o + i) = make_float4(p.keep * acc[i] + add, p.keep * acc[i + 1] + add,
                                                        p.keep * acc[i + 2] + add, p.keep * acc[i + 3] + add);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// Output GEMM of the band interpolation with 256-column tiles:
// out(y, g * 256 + j) = osc * sum_k P(y, k) Z(g * 256 + j, k) over hi/lo
// planes (hi.hi + hi.lo + lo.hi): FP16 with osc = interp_scale(mean) for the
// separable form (p.f16, p.mean), BF16 with osc = 1 for the Hermitian
// half-band operands.  P's 128-row tile stays resident in shared memory in
// ABOX 32-wide boxes per plane (64B swizzle, 8 KB each: 80 KB at K = 160);
// Z's 256-row tiles stream through a ring of STAGES stages, one plane of one
// 32-wide box each (16 KB; the hi plane feeds hi.hi and lo.hi, the lo plane
// hi.lo), so each MMA is 128 x 256 x 16.  The kernel is bound by how much
// of Z is in flight: at M = 160 and 256 clips 4 / 5 / 6 / 7 stages of 16 KB
// take 0.363 / 0.340 / 0.316 / 0.300 ms (3 stages of both planes, 32 KB
// each: 0.317 ms); more staging tiles per epilogue warp than two do not help.
// Accumulators double-buffered in all 512 TMEM columns.  Roles as
// tc_dft_gemm MODE 1 (warp 0 TMA, warp 1 MMA issue, warps 2-5 epilogue with
// TMA stores).  grid: (1, a_rows / 128, problems); p.G = out columns / 256,
// p.kboxes = 32-wide A boxes.
constexpr uint32_t kW256ABox = 128 * 64;  // one plane: 128 rows x 32 fp16
constexpr uint32_t kW256BBox = 256 * 64;  // one plane: 256 rows x 32 fp16
__host__ __device__ constexpr size_t w256_smem_bytes(int abox, int stages, int outbufs) {
  return 1024 + 2 * static_cast<size_t>(abox) * kW256ABox + static_cast<size_t>(stages) * kW256BBox +
         4 * static_cast<size_t>(outbufs) * kOutTile + 256;
}
// K <= 160 (ten 16-wide K steps) and K <= 192
static_assert(w256_smem_bytes(5, 7, 2) <= 232448, "tc_interp_w256: more shared memory than one CTA may have");
static_assert(w256_smem_bytes(6, 6, 2) <= 232448, "tc_interp_w256: more shared memory than one CTA may have");

template <int ABOX, int STAGES, int OUTBUFS>
__global__ void __launch_bounds__(192, 1)
    tc_interp_w256(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ CUtensorMap tmO, TcGemmParams p) {
  constexpr int kW256Stages = STAGES, kW256OutBufs = OUTBUFS;
  constexpr uint32_t kTmemCols = 512;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  uint8_t* sA = base;                                    // [plane][ABOX boxes] x 8 KB
  uint8_t* sB = sA + 2 * ABOX * kW256ABox;               // [stage] x 16 KB (one plane)
  uint8_t* sO = sB + kW256Stages * kW256BBox;            // epilogue staging
  uint64_t* bars = reinterpret_cast<uint64_t*>(sO + 4 * kW256OutBufs * kOutTile);
  uint64_t* full = bars;
  uint64_t* empty = bars + kW256Stages;
  uint64_t* a_full = bars + 2 * kW256Stages;
  uint64_t* tfull = bars + 2 * kW256Stages + 1;
  uint64_t* tempty = bars + 2 * kW256Stages + 3;
  uint64_t* done = bars + 2 * kW256Stages + 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kW256Stages + 6);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m_tile = blockIdx.y, prob = blockIdx.z;
  const int kbb = (p.ksteps + 1) / 2;  // 32-wide B boxes per step

  if (threadIdx.x == 0) {
    for (int s = 0; s < kW256Stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(a_full, 1);
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

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&tmA);
      prefetch_tmap(&tmB);
      mbar_arrive_expect_tx(a_full, 2u * p.kboxes * kW256ABox);
      for (int part = 0; part < 2; ++part)
        for (int kb = 0; kb < p.kboxes; ++kb)
          tma_load_2d(sA + (part * ABOX + kb) * kW256ABox, &tmA, kb * 32, part * p.a_rows + m_tile * 128, a_full);
      int it = 0;
      for (int g = 0; g < p.G && !*abort_flag; ++g) {
        bool ok = true;
        for (int kb = 0; kb < kbb && ok; ++kb)
          for (int pl = 0; pl < 2; ++pl, ++it) {
            const int s = it % kW256Stages;
            const uint32_t ph = (it / kW256Stages) & 1;
            if (!mbar_wait_or_abort(&empty[s], ph ^ 1, kWaitLimitNs, abort_flag)) {
              fail(21);
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&full[s], kW256BBox);
            const int row = prob * p.b_prob + g * 256 + pl * p.b_plane;
            tma_load_2d(sB + s * kW256BBox, &tmB, kb * 32, row, &full[s]);
          }
        if (!ok) break;
      }
      // Drain: every load issued must have landed before the CTA may exit.
      mbar_wait(a_full, 0, kWaitLimitNs);
      for (int q = (it > kW256Stages ? it - kW256Stages : 0); q < it; ++q)
        mbar_wait(&full[q % kW256Stages], (q / kW256Stages) & 1, kWaitLimitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = p.f16 ? idesc_f16(128, 256) : idesc_bf16(128, 256);
      bool ok = mbar_wait(a_full, 0, kWaitLimitNs);
      if (!ok) fail(22);
      if (ok && p.probe_wait_ns && !mbar_wait(done, 0, p.probe_wait_ns)) {  // nothing arrives at `done` yet
        fail(26);
        ok = false;
      }
      tc_fence_after();
      int it = 0;
      for (int g = 0; g < p.G && ok && !*abort_flag; ++g) {
        const int buf = g & 1;
        if (!mbar_wait_or_abort(&tempty[buf], ((g >> 1) & 1) ^ 1, kWaitLimitNs, abort_flag)) {
          fail(23);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + buf * 256;
        for (int kb = 0; kb < kbb && ok; ++kb)
          for (int pl = 0; pl < 2; ++pl, ++it) {
            const int s = it % kW256Stages;
            if (!mbar_wait(&full[s], (it / kW256Stages) & 1, kWaitLimitNs)) {
              fail(24);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t b = smem_desc_sw64(smem_u32(sB + s * kW256BBox));
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const int kstep = kb * 2 + ks;
              if (kstep < p.ksteps) {
                // A: 32-wide box kstep / 2 (= kb), 32 bytes per 16-wide K step inside it
                const uint64_t a_hi = smem_desc_sw64(smem_u32(sA + (0 * ABOX + kb) * kW256ABox)) +
                                      static_cast<uint64_t>(2 * ks);
                const uint64_t a_lo = smem_desc_sw64(smem_u32(sA + (1 * ABOX + kb) * kW256ABox)) +
                                      static_cast<uint64_t>(2 * ks);
                const uint64_t adv = static_cast<uint64_t>(2 * ks);
                if (pl == 0) {  // hi plane of B: hi.hi and lo.hi
                  tc_mma_bf16(d, a_hi, b + adv, idesc, kstep > 0 ? 1u : 0u);
                  tc_mma_bf16(d, a_lo, b + adv, idesc, 1u);
                } else {  // lo plane of B: hi.lo
                  tc_mma_bf16(d, a_hi, b + adv, idesc, 1u);
                }
              }
            }
            tc_commit(&empty[s]);
          }
        if (!ok) break;
        tc_commit(&tfull[buf]);
      }
      // All MMAs issued by this thread have completed once `done` flips.
      tc_commit(done);
      mbar_wait(done, 0, kWaitLimitNs);
    }
  } else {
    // Epilogue warps 2..5: TMEM lane quadrant = warp % 4.
    const int quad = warp & 3;
    const float osc = p.mean ? interp_scale(p.mean[prob]) : 1.f;
    int nst = 0;  // TMA-store tiles issued by this warp
    for (int g = 0; g < p.G; ++g) {
      const int buf = g & 1;
      // Warp-uniform outcome: tcgen05.ld below is .sync.aligned.
      const bool got = __all_sync(0xffffffffu, mbar_wait_or_abort(&tfull[buf], (g >> 1) & 1, kWaitLimitNs, abort_flag));
      if (!got) {
        if (lane == 0) fail(25);
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16) + buf * 256;
#pragma unroll 1
      for (int c0 = 0; c0 < 256; c0 += 32) {
        float v[32];
        tmem_ld32(taddr + c0, v);
        // buffer `sb` was last read by the store issued kW256OutBufs tiles ago
        const int sbuf = nst % kW256OutBufs;
        if (lane == 0 && nst >= kW256OutBufs) bulk_wait_read<kW256OutBufs - 1>();
        __syncwarp();
        uint8_t* sb = sO + (quad * kW256OutBufs + sbuf) * kOutTile;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          *reinterpret_cast<float4*>(sb + lane * 128 + ((q ^ (lane & 7)) << 4)) =
              make_float4(osc * v[4 * q], osc * v[4 * q + 1], osc * v[4 * q + 2], osc * v[4 * q + 3]);
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          tma_store_2d(&tmO, sb, g * 256 + c0, prob * p.a_rows + m_tile * 128 + quad * 32);
          bulk_commit();
        }
        ++nst;
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
    // Every TMA store must have finished before the CTA's shared memory goes.
    if (lane == 0 && nst > 0) bulk_wait<0>();
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// Row transform along x of the band products, written as the tensor-core
// B operand: Bop[problem][k][plane][x][kk], kk = 2 * (row - row_off) + re/im,
// planes hi / lo, K-major with row stride kp.  Rows [row_off, row_off + nrows)
// of the band are used.  Columns [2 * nrows, zero_to) are written as zeros.
// grid: (ceil(K * nrows / S), problems).
__global__ void socs_rows_tc(const float2* __restrict__ kband, float scale, const float2* __restrict__ Mband,
                             int K, int hb, int row_off, int nrows, int lg, int S, int kp, int zero_to,
                             __nv_bfloat16* __restrict__ Bop, const float2* __restrict__ tw) {
  extern __shared__ float2 smem[];
  const int L = 1 << lg;
  const int B = 2 * hb + 1;
  const int prob = blockIdx.y;
  const int seq0 = blockIdx.x * S;
  const int nseq = min(S, K * nrows - seq0);
  float2* a = smem;
  float2* b = smem + (S << lg);
  for (int t = threadIdx.x; t < (S << lg); t += blockDim.x) a[t] = make_float2(0.f, 0.f);
  __syncthreads();
  const float2* Mc = Mband + static_cast<size_t>(prob) * B * B;
  for (int t = threadIdx.x; t < nseq * B; t += blockDim.x) {
    const int s = t / B, mx = t - s * B;
    const int seq = seq0 + s;
    const int k = seq / nrows, my = row_off + (seq - k * nrows);
    const float2 m = Mc[static_cast<size_t>(my) * B + mx];
    const float2 u = kband ? kband[(static_cast<size_t>(k) * B + my) * B + mx] : make_float2(scale, 0.f);
    a[(s << lg) + ((mx - hb) & (L - 1))] = cmul(u, m);
  }
  __syncthreads();
  const float2* r = block_fft<+1>(a, b, lg, S, tw);
  const size_t plane = static_cast<size_t>(L) * kp;
  for (int t = threadIdx.x; t < (nseq << lg); t += blockDim.x) {
    const int s = t % nseq, x = t / nseq;
    const int seq = seq0 + s;
    const int k = seq / nrows, myr = seq - k * nrows;
    const float2 v = r[(s << lg) + x];
    __nv_bfloat16 rh, rl, ih, il;
    split_bf16(v.x, rh, rl);
    split_bf16(v.y, ih, il);
    __nv_bfloat16* hi = Bop + (static_cast<size_t>(prob) * K + k) * 2 * plane + static_cast<size_t>(x) * kp;
    __nv_bfloat16* lo = hi + plane;
    __nv_bfloat162 hv, lv;
    hv.x = rh;
    hv.y = ih;
    lv.x = rl;
    lv.y = il;
    *reinterpret_cast<__nv_bfloat162*>(hi + 2 * myr) = hv;
    *reinterpret_cast<__nv_bfloat162*>(lo + 2 * myr) = lv;
    if (myr == nrows - 1) {
      const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
      for (int kk = 2 * nrows; kk < zero_to; ++kk) {
        hi[kk] = z;
        lo[kk] = z;
      }
    }
  }
}

// socs_rows_tc with register-radix passes (fft_reg.cuh): S sequences of
// length L = 2^LG per block, one radix-16 butterfly per thread per pass.  The
// band products are read once into a compact [S][B] array, the first pass
// reads them as the zero-padded band, and the last pass writes the split
// operand straight from registers (consecutive lanes = consecutive band rows
// of one x, so each store covers contiguous words).
// grid: (ceil(K * nrows / S), problems); block fr_threads(L, S).
template <int L, int S>
__global__ void __launch_bounds__(fr_threads(L, S))
    socs_rows_reg(const float2* __restrict__ kband, float scale, const float2* __restrict__ Mband, int K, int hb,
                  int row_off, int nrows, int kp, int zero_to, __nv_bfloat16* __restrict__ Bop,
                  const float2* __restrict__ tw) {
  constexpr int T = fr_threads(L, S), NP = fr_passes(L);
  constexpr int R = fr_radix(L, NP - 1);
  extern __shared__ float2 smem[];
  const int B = 2 * hb + 1;
  const int prob = blockIdx.y;
  const int seq0 = blockIdx.x * S;
  const int nseq = min(S, K * nrows - seq0);
  const int t = threadIdx.x;
  float2* P = smem;  // [S][B]
  float2* b0 = smem + S * B;
  float2* b1 = b0 + fr_buf(L, S);
  const float2* Mc = Mband + static_cast<size_t>(prob) * B * B;
  // one warp per sequence: (k, my) once per row, lanes along mx (no divisions)
  for (int s = t >> 5; s < S; s += T / 32) {
    float2* Ps = P + s * B;
    if (s < nseq) {
      const int seq = seq0 + s;
      const int k = seq / nrows, my = row_off + (seq - k * nrows);
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
    fr_mid_pass<L, S, +1, 1>(t, b0, b1, tw);
    __syncthreads();
    src = b1;
  }
  const size_t plane = static_cast<size_t>(L) * kp;
#pragma unroll
  for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
    if (t + b * T >= fr_nb(L, S, NP - 1)) break;
    int s, j;
    float2 v[R];
    fr_last_pass<L, S, +1>(t + b * T, src, tw, s, j, v);
    if (s >= nseq) continue;
    const int seq = seq0 + s;
    const int k = seq / nrows, myr = seq - k * nrows;
    __nv_bfloat16* hi = Bop + (static_cast<size_t>(prob) * K + k) * 2 * plane + 2 * myr;
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const size_t x = static_cast<size_t>(j + p * (L / R));
      // (re, im) -> bf16x2 hi, then the packed residual as lo
      const __nv_bfloat162 hv = __float22bfloat162_rn(v[p]);
      const float2 hf = __bfloat1622float2(hv);
      const __nv_bfloat162 lv = __float22bfloat162_rn(make_float2(v[p].x - hf.x, v[p].y - hf.y));
      *reinterpret_cast<__nv_bfloat162*>(hi + x * kp) = hv;
      *reinterpret_cast<__nv_bfloat162*>(hi + plane + x * kp) = lv;
    }
    if (myr == nrows - 1) {
      const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
      for (int p = 0; p < R; ++p) {
        __nv_bfloat16* row = hi - 2 * myr + static_cast<size_t>(j + p * (L / R)) * kp;
        for (int kk = 2 * nrows; kk < zero_to; ++kk) {
          row[kk] = z;
          row[plane + kk] = z;
        }
      }
    }
  }
}

// Sequences per block of socs_rows_reg for L = 2^lg (0: no instance).
constexpr int rows_reg_S(int L) { return xt_S(L); }
constexpr size_t rows_reg_smem(int L, int B) {
  return (static_cast<size_t>(rows_reg_S(L)) * B +
          (fr_passes(L) - 1) * static_cast<size_t>(fr_buf(L, rows_reg_S(L)))) *
         sizeof(float2);
}

// Band products of every kernel with the mask band, split into BF16 planes as
// the B operand of the row-transform GEMM: P[prob][k][plane][my][kk], rows my
// padded to rows_pad, kk = 2 mx + re/im padded to kp; zero outside my < B,
// mx < B.  grid (K, problems).
__global__ void band_products(const float2* __restrict__ kband, const float2* __restrict__ Mband, int K, int B,
                              int rows_pad, int kp, __nv_bfloat16* __restrict__ P) {
  const int k = blockIdx.x, prob = blockIdx.y;
  const float2* Mc = Mband + static_cast<size_t>(prob) * B * B;
  const float2* u = kband + static_cast<size_t>(k) * B * B;
  const size_t plane = static_cast<size_t>(rows_pad) * kp;
  __nv_bfloat162* hi = reinterpret_cast<__nv_bfloat162*>(P + (static_cast<size_t>(prob) * K + k) * 2 * plane);
  __nv_bfloat162* lo = hi + plane / 2;
  const int pairs = kp / 2;
  for (int e = threadIdx.x; e < rows_pad * pairs; e += blockDim.x) {
    const int my = e / pairs, mx = e - my * pairs;
    __nv_bfloat162 h, l;
    h.x = h.y = l.x = l.y = __float2bfloat16_rn(0.f);
    if (my < B && mx < B) {
      const float2 v = cmul(u[my * B + mx], Mc[my * B + mx]);
      split_bf16(v.x, h.x, l.x);
      split_bf16(v.y, h.y, l.y);
    }
    hi[e] = h;
    lo[e] = l;
  }
}

}  // namespace huv_dev

// ------------------------------------------------------------------ host
namespace huv_launch {

using namespace huv_dev;

// Length of the probe wait the tensor-core kernels take before their first
// MMA (0 = none); set by huv_debug_probe_wait for tests of the give-up path.
std::atomic<unsigned long long> g_probe_wait_ns{0};
size_t field_fused_part_bytes(int L, int K);
cudaError_t socs_field_fused(const float2* kband, const float2* Mband, int K, int hb, int L, int clips, float keep,
                             float flare, const float* mean, float* out, void* split, float* part, const float2* tw,
                             cudaStream_t st);
unsigned long long probe_wait_ns() { return g_probe_wait_ns.load(std::memory_order_relaxed); }
bool xt_ok(int L, int hb);
cudaError_t socs_rows_x(const float2* kband, float scale, const float2* Mband, int K, int hb, int L, int clips,
                        float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols_x(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                        const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
cudaError_t socs_cols_split(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                            const float* mean, void* split, const float2* tw, cudaStream_t st);

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// 2-D bf16 tensor map over a K-major [rows][kp] array, box 64 x box_rows, 128B swizzle.
// With cols > 0 the map ends at column cols (< kp): TMA fills the columns
// beyond it with zeros instead of reading them.
bool make_map(CUtensorMap* map, const void* ptr, uint64_t rows, int kp, int box_rows, int cols = 0,
              bool f16 = false) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols > 0 ? cols : kp), rows};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(kp) * 2};
  cuuint32_t box[2] = {64, static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr),
            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D fp16 / bf16 tensor map (box 32 x box_rows, 64B swizzle) over
// [rows][cols], row stride kp elements: the 128-row A and 256-row B tiles of
// tc_interp_w256.
bool make_map_sw64(CUtensorMap* map, const void* ptr, uint64_t rows, int kp, int box_rows, int cols, bool f16) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), rows};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(kp) * 2};
  cuuint32_t box[2] = {32, static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D f32 tensor map over [rows][cols] (row stride cols floats), 32 x 32
// boxes with 128B swizzle: the TMA-store target of the interpolation GEMM.
bool make_out_map(CUtensorMap* map, void* ptr, uint64_t rows, uint64_t cols) {
  auto fn = encode_fn();
  if (!fn || (reinterpret_cast<uintptr_t>(ptr) & 15u) != 0 || (cols * 4) % 16 != 0) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 4};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

uint16_t host_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t rounding = 0x7FFFu + ((u >> 16) & 1u);
  return static_cast<uint16_t>((u + rounding) >> 16);
}
float host_bf16_to_f(uint16_t h) {
  const uint32_t u = static_cast<uint32_t>(h) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// FP16 split planes [2][rows][kp] (hi, lo = the FP32 remainder rounded to FP16)
// of a real matrix given row-major values [rows][kc].
std::vector<uint16_t> split_planes_f16(const std::vector<double>& v, int rows, int kc, int kp) {
  std::vector<uint16_t> out(2 * static_cast<size_t>(rows) * kp, 0);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < kc; ++c) {
      const float f = static_cast<float>(v[static_cast<size_t>(r) * kc + c]);
      const __half hi = __float2half_rn(f);
      const __half lo = __float2half_rn(f - __half2float(hi));
      out[static_cast<size_t>(r) * kp + c] = static_cast<__half_raw>(hi).x;
      out[(static_cast<size_t>(rows) + r) * kp + c] = static_cast<__half_raw>(lo).x;
    }
  return out;
}

// Split planes [2][rows][kp] of a real matrix given row-major values [rows][kc].
std::vector<uint16_t> split_planes(const std::vector<double>& v, int rows, int kc, int kp) {
  std::vector<uint16_t> out(2 * static_cast<size_t>(rows) * kp, 0);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < kc; ++c) {
      const float f = static_cast<float>(v[static_cast<size_t>(r) * kc + c]);
      const uint16_t hi = host_bf16(f);
      const uint16_t lo = host_bf16(f - host_bf16_to_f(hi));
      out[static_cast<size_t>(r) * kp + c] = hi;
      out[(static_cast<size_t>(rows) + r) * kp + c] = lo;
    }
  return out;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Row transforms into the split operand: register-radix kernel for
// L = 128 .. 1024 (band within 110 KiB of shared memory), else the
// shared-memory radix-4 kernel.
void launch_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int row_off, int nrows,
                 int L, int kp, int zero_to, __nv_bfloat16* Bop, const float2* tw, int problems, cudaStream_t st) {
  const int B = 2 * hb + 1;
  const int S = rows_reg_S(L);
  const bool inst = L == 128 || L == 160 || L == 192 || L == 256 || L == 512 || L == 1024;  // the instances below
  if (S > 0 && inst && 2 * hb < L && rows_reg_smem(L, B) <= 110 * 1024) {
    const dim3 g((K * nrows + S - 1) / S, problems);
    const size_t sm = rows_reg_smem(L, B);
    switch (L) {
      case 128: socs_rows_reg<128, 32><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;
      case 160: socs_rows_reg<160, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;
      case 192: socs_rows_reg<192, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;
      case 256: socs_rows_reg<256, 16><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;
      case 512: socs_rows_reg<512, 8><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;
      default: socs_rows_reg<1024, 4><<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, kp, zero_to, Bop, tw); break;  // L == 1024
    }
    return;
  }
  int lg = 0;
  while ((1 << lg) < L) ++lg;
  const int S8 = fit_units(8, 2 * (sizeof(float2) << lg));
  const dim3 g((K * nrows + S8 - 1) / S8, problems);
  const size_t sm = 2 * (static_cast<size_t>(S8) << lg) * sizeof(float2);
  socs_rows_tc<<<g, 256, sm, st>>>(kband, scale, Mband, K, hb, row_off, nrows, lg, S8, kp, zero_to, Bop, tw);
}

}  // namespace

// 2-D bf16 tensor map (box 64 x box_rows, 128B swizzle) for other files' kernels.
bool tc_map_bf16(CUtensorMap* map, const void* ptr, uint64_t rows, int kp, int box_rows) {
  return make_map(map, ptr, rows, kp, box_rows);
}

cudaError_t tc_set_smem() {
  const int bytes = static_cast<int>(tc_smem_bytes(3));
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(3, kTcBN, false, true)))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<2, kRowBN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(3, kRowBN, true)))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<2, kRowBNWide>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(3, kRowBNWide, true)))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_interp_w256<5, 7, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(w256_smem_bytes(5, 7, 2)))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_interp_w256<6, 6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(w256_smem_bytes(6, 6, 2)))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<3, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(2, 64, false, false, tc_stages(3, 64))))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<3, 80>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(3, 80, false, false, tc_stages(3, 80))))))
    return e;
  if ((e = cudaFuncSetAttribute(tc_dft_gemm<3, 96>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tc_smem_bytes(3, 96, false, false, tc_stages(3, 96))))))
    return e;
  if ((e = cudaFuncSetAttribute(socs_rows_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  const int reg_bytes = 110 * 1024;
#define HUV_ROWS_ATTR(LL, SS)                                                                                \
  if ((e = cudaFuncSetAttribute(socs_rows_reg<LL, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, reg_bytes))) \
    return e;
  HUV_ROWS_ATTR(128, 32) HUV_ROWS_ATTR(160, 16) HUV_ROWS_ATTR(192, 16) HUV_ROWS_ATTR(256, 16)
  HUV_ROWS_ATTR(512, 8) HUV_ROWS_ATTR(1024, 4)
#undef HUV_ROWS_ATTR
  return cudaSuccess;
}

void tc_release(huv::TcState& tc) {
  cudaFree(tc.gy);
  cudaFree(tc.gx);
  cudaFree(tc.gp);
  tc = huv::TcState();
}

void tc_release_all(std::map<int, huv::TcState>& m) {
  for (auto& kv : m) tc_release(kv.second);
  m.clear();
}

}  // namespace huv_launch

namespace huv {

namespace {
constexpr double kPi = 3.14159265358979323846;
inline int ilog2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
}  // namespace

bool Engine::hybrid_supported(const DeviceSet& ds, int M) const {
  const int kpI = ((2 * (2 * ds.hb + 1)) + 63) / 64 * 64;
  const bool pow2 = (M & (M - 1)) == 0;
  return n >= 128 && n % 128 == 0 && M <= n && kpI <= 192 && huv_launch::encode_fn() != nullptr &&
         (pow2 || (huv_launch::xt_ok(M, ds.hb) && huv_launch::xt_ok(M, 2 * ds.hb)));
}

bool Engine::tc_supported(const DeviceSet& ds, int M) const {
  const int kpE = ((2 * ds.B) + 63) / 64 * 64;
  const int kpI = ((2 * (2 * ds.hb + 1)) + 63) / 64 * 64;
  return M >= 128 && n >= 128 && M % huv_dev::kTcBN == 0 && kpE <= 192 && kpI <= 192 &&
         huv_launch::encode_fn() != nullptr;
}

void Engine::run_tc_form(const huv_batch& b, DeviceSet& ds, int M, float* out, cudaStream_t st, int K_use,
                         const float* W_use, int core) {
  const bool gemm_rows = core == kTcCoreGemmRows, fft_field = core == kTcCoreFftField;
  using namespace huv_launch;
  static std::atomic<uint64_t> smem_set{0};
  once_per_device(smem_set, [] { check_cuda(tc_set_smem(), "cudaFuncSetAttribute(tc)"); });
  const int lgn = ilog2i(n), lgm = ilog2i(M);  // lgm: log2 of M rounded up (M need not be a power of two)
  const int B = ds.B, K = K_use > 0 ? K_use : ds.K, hb = ds.hb;
  const float* Wf = W_use ? W_use : ds.W;
  const int h2 = 2 * hb, B2 = 2 * h2 + 1;
  const int kcE = 2 * B, kpE = round_up(kcE, 64), kstE = (kcE + 15) / 16;
  const int nrI = h2 + 1, kcI = 2 * nrI, kpI = round_up(kcI, 64), kstI = (kcI + 15) / 16;
  // The split operands written per chunk are laid out with rows of the K
  // extent the MMAs read (16 ksteps) and written only up to the band's
  // 2 B columns: their tensor maps end at column 2 B, so TMA fills the rest
  // of the last 64-wide box with zeros instead of reading padding.
  const int kbE = kstE * 16, kbI = kstI * 16;
  // Separable interpolation (evaluation grids up to 192 points, FP32 field
  // pass): the coarse intensity is band-limited to |f| <= h2 < M / 2, so
  // I_N = P I_M P^T exactly, with the real N x M matrix
  //     P(Y, m) = (1/M) sum_{|f| <= h2} exp(2 pi i f (Y/N - m/M))
  // (a Dirichlet kernel).  Z^T = P I_M^T is one small tcgen05 GEMM (MODE 3,
  // split operand out) and I_N = P Z the store-mode GEMM (MODE 1), in place
  // of the band transform of I_M and the N-point row transforms.  Operands
  // are FP16 hi/lo planes (22 significant bits against BF16's 16) with I_M
  // carried as I_M / interp_scale(mean); the final GEMM multiplies it back.
  const bool sep = fft_field && M <= 192 && M % 16 == 0 && xt_ok(M, hb);
  TcState& tc = ds.tc[M];
  if (sep) interp_matrix(ds, M);
  if (!fft_field && !tc.gy) {
    // A_E: rows (y, re/im) over the M grid, K = (my, re/im).
    std::vector<double> ae(static_cast<size_t>(2 * M) * kcE);
    for (int y = 0; y < M; ++y)
      for (int mi = 0; mi < B; ++mi) {
        const double th = 2.0 * kPi * (mi - hb) * static_cast<double>(y) / M;
        const double c = std::cos(th), s = std::sin(th);
        double* re = &ae[static_cast<size_t>(2 * y) * kcE];
        double* im = &ae[static_cast<size_t>(2 * y + 1) * kcE];
        re[2 * mi] = c;
        re[2 * mi + 1] = -s;
        im[2 * mi] = s;
        im[2 * mi + 1] = c;
      }
    const auto pe = split_planes(ae, 2 * M, kcE, kpE);
    check_cuda(cudaMalloc(&tc.gy, pe.size() * 2), "cudaMalloc(A_E)");
    check_cuda(cudaMemcpy(tc.gy, pe.data(), pe.size() * 2, cudaMemcpyHostToDevice), "upload A_E");
    if (!make_map(&tc.map_ae, tc.gy, 2ull * 2 * M, kpE, 128))
      throw Error(HUV_ERR_CUDA, "cuTensorMapEncodeTiled failed for the DFT operands");
  }
  if (!tc.gx) {
    // A_I: rows y over the N grid, K = (qy >= 0, re/im), Hermitian weights.
    std::vector<double> ai(static_cast<size_t>(n) * kcI);
    for (int y = 0; y < n; ++y)
      for (int q = 0; q <= h2; ++q) {
        const double th = 2.0 * kPi * q * static_cast<double>(y) / n;
        const double w = q == 0 ? 1.0 : 2.0;
        ai[static_cast<size_t>(y) * kcI + 2 * q] = w * std::cos(th);
        ai[static_cast<size_t>(y) * kcI + 2 * q + 1] = -w * std::sin(th);
      }
    const auto pi = split_planes(ai, n, kcI, kpI);
    check_cuda(cudaMalloc(&tc.gx, pi.size() * 2), "cudaMalloc(A_I)");
    check_cuda(cudaMemcpy(tc.gx, pi.data(), pi.size() * 2, cudaMemcpyHostToDevice), "upload A_I");
    if (!make_map(&tc.map_ai, tc.gx, 2ull * n, kpI, 128) ||
        !make_map_sw64(&tc.map_ai32, tc.gx, 2ull * n, kpI, 128, kpI, false))
      throw Error(HUV_ERR_CUDA, "cuTensorMapEncodeTiled failed for the DFT operands");
    tc.lgm = lgm;
  }
  const size_t in_elem = b.input_kind == HUV_INPUT_RASTER_U8
                             ? 1
                             : (b.input_kind == HUV_INPUT_RASTER_F32 ? 4 : (b.input_kind == HUV_INPUT_RECTS ? 0 : 8));
  const size_t per_x = align256(sizeof(float2) * n * B);
  const size_t per_m = align256(sizeof(float2) * B * B);
  const bool fused = fft_field && field_fused(ds, M);
  const size_t per_be = align256(std::max(static_cast<size_t>(K) * 2 * M * kbE * 2,
                                          fused ? field_fused_part_bytes(M, K) : size_t(0)));
  const int rbn = B <= kRowBN ? kRowBN : kRowBNWide;  // rows of P (band rows my, padded)
  if (gemm_rows && B > kRowBNWide) throw Error(HUV_ERR_UNSUPPORTED, "TC form: band wider than 96 orders");
  const size_t per_p = gemm_rows ? align256(static_cast<size_t>(K) * 2 * rbn * kpE * 2) : 0;
  const size_t per_i = align256(sizeof(float) * M * M);
  const size_t per_x2 = sep ? 0 : align256(sizeof(float2) * M * B2);  // band of I_M (band-transform path)
  const size_t per_c = sep ? 0 : align256(sizeof(float2) * B2 * B2);
  const size_t per_bi = align256(static_cast<size_t>(2) * n * std::max(kbI, M) * 2);
  const size_t per_mean = align256(sizeof(float) * (1 + (B + 3) / 4));
  const size_t per_clip = per_x + per_m + per_be + per_p + per_i + per_x2 + per_c + per_bi + per_mean;
  // a C2 step (256 clips) runs as one chunk of the engine's own workspace, so
  // the column pass (2 blocks per SM, 10 blocks per clip) fills whole waves
  const size_t budget = chunk_budget();
  const int chunk = balanced_chunk(static_cast<int>(std::max<size_t>(1, budget / per_clip)), b.n_clips);
  char* base = static_cast<char*>(workspace(per_clip * chunk + 4096));
  size_t off = 0;
  auto take = [&](size_t per) {
    char* p = base + off;
    off += per * chunk;
    return p;
  };
  float2* X = reinterpret_cast<float2*>(take(per_x));
  float2* Mb = reinterpret_cast<float2*>(take(per_m));
  __nv_bfloat16* BE = reinterpret_cast<__nv_bfloat16*>(take(per_be));
  __nv_bfloat16* P = reinterpret_cast<__nv_bfloat16*>(take(per_p));
  float* IM = reinterpret_cast<float*>(take(per_i));
  float2* X2 = reinterpret_cast<float2*>(take(per_x2));
  float2* C = reinterpret_cast<float2*>(take(per_c));
  __nv_bfloat16* BI = reinterpret_cast<__nv_bfloat16*>(take(per_bi));
  float* mean = reinterpret_cast<float*>(take(per_mean));
  const float2* twn = twiddle_n(n);
  const float2* twm = twiddle_n(M);
  const size_t smem_tc = tc_smem_bytes(3);
  for (int c0 = 0; c0 < b.n_clips; c0 += chunk) {
    const int nc = std::min(chunk, b.n_clips - c0);
    const void* in = static_cast<const char*>(b.input) + in_elem * static_cast<size_t>(n) * n * c0;
    float* o = out + static_cast<size_t>(n) * n * c0;
    prof.begin("mask_band", st);
    if (b.input_kind == HUV_INPUT_RECTS)
      rect_band(c0, nc, hb, Wf, Mb, mean, st);  // host-side table, exact spectrum on the device
    else
      check_cuda(band_forward(in, b.input_kind, n, lgn, hb, nc, X, Mb, b.pixel_transfer ? ds.ptx : nullptr, Wf,
                              mean, twn, st, row_digit_table(hb), dev_err),
                 "band_forward");
    prof.end(st);
    CUtensorMap mbE, mbI, mbP;
    if (!make_map(&mbE, BE, static_cast<uint64_t>(nc) * K * 2 * M, kbE, kTcBN, kcE) ||
        !make_map(&mbI, BI, static_cast<uint64_t>(nc) * 2 * n, kbI, kTcBN, kcI) ||
        (gemm_rows && !make_map(&mbP, P, static_cast<uint64_t>(nc) * K * 2 * rbn, kpE, rbn)))
      throw Error(HUV_ERR_CUDA, "cuTensorMapEncodeTiled failed for the band operands");
    if (fft_field) {
      // FP32 register-radix field pass: rows x-major into the operand
      // buffer (K B M complex fits in its K 2 M kbE bf16), columns with
      // sum lambda |E|^2 in registers, normalisation and flare -> IM
      float2* T = reinterpret_cast<float2*>(BE);
      if (fused) {
        // one kernel per kernel group: rows and columns in shared memory; the
        // groups' partial sums (if any) in the operand buffer
        prof.begin("socs_field_fused", st);
        check_cuda(socs_field_fused(ds.kband, Mb, K, hb, M, nc, ds.keep, ds.flare, mean, sep ? nullptr : IM,
                                    sep ? static_cast<void*>(IM) : nullptr, reinterpret_cast<float*>(BE), twm, st),
                   "socs_field_fused");
        prof.end(st);
      } else {
        prof.begin("socs_rows_inv", st);
        check_cuda(socs_rows_x(ds.kband, 0.f, Mb, K, hb, M, nc, T, twm, st), "socs_rows");
        prof.end(st);
        prof.begin("socs_cols_inv", st);
        if (sep)  // I_M / s as FP16 split planes [clip][2][M][M] (the bytes of the f32 IM)
          check_cuda(socs_cols_split(T, K, hb, M, nc, ds.keep, ds.flare, mean, IM, twm, st), "socs_cols");
        else
          check_cuda(socs_cols_x(T, K, hb, M, nc, ds.keep, ds.flare, mean, IM, 0, twm, st), "socs_cols");
        prof.end(st);
      }
    }
    if (!fft_field) prof.begin(gemm_rows ? "tc_dft_gemm<rows>" : "socs_rows_tc", st);
    if (fft_field) {
    } else if (!gemm_rows) {
      // Row transforms as FP32 register-radix FFTs, emitting the split operand.
      launch_rows(ds.kband, 0.f, Mb, K, hb, 0, B, M, kbE, 0, BE, twm, nc, st);
      check_cuda(cudaGetLastError(), "socs_rows_tc");
    } else {
      // Row transforms of every kernel's band product on tensor cores: the
      // same M-point inverse DFT operand (A_E) against the split products,
      // written straight as the next GEMM's split operand.
      band_products<<<dim3(K, nc), 256, 0, st>>>(ds.kband, Mb, K, B, rbn, kpE, P);
      check_cuda(cudaGetLastError(), "band_products");
      TcGemmParams p{};
      p.kboxes = kpE / 64;
      p.ksteps = kstE;
      p.G = K;
      p.a_rows = 2 * M;
      p.b_prob = K * 2 * rbn;
      p.b_step = 2 * rbn;
      p.b_plane = rbn;
      p.err = dev_err;
      p.probe_wait_ns = huv_launch::probe_wait_ns();
      p.bop = BE;
      p.bop_g = 2ll * M * kbE;
      p.bop_prob = static_cast<long long>(K) * 2 * M * kbE;
      p.bop_plane = static_cast<long long>(M) * kbE;
      p.bop_ld = kbE;
      p.bop_cols = std::min(kstE * 8, rbn);  // the K columns GEMM0 reads: 2 my + re/im < 16 kstE
      dim3 g(1, 2 * M / 128, nc);
      if (rbn == kRowBN)
        tc_dft_gemm<2, kRowBN><<<g, 192, tc_smem_bytes(3, kRowBN, true), st>>>(tc.map_ae, mbP, tc.map_ae, p);
      else
        tc_dft_gemm<2, kRowBNWide>
            <<<g, 192, tc_smem_bytes(3, kRowBNWide, true), st>>>(tc.map_ae, mbP, tc.map_ae, p);
      check_cuda(cudaGetLastError(), "tc_dft_gemm<2>");
    }
    if (!fft_field) prof.end(st);
    if (!fft_field) {
      TcGemmParams p{};
      p.kboxes = kpE / 64;
      p.ksteps = kstE;
      p.G = K;
      p.a_rows = 2 * M;
      p.b_prob = K * 2 * M;
      p.b_step = 2 * M;
      p.b_plane = M;
      p.out_ld = M;
      p.out_plane = static_cast<long long>(M) * M;
      p.keep = ds.keep;
      p.flare = ds.flare;
      p.mean = mean;
      p.out = IM;
      p.err = dev_err;
      p.probe_wait_ns = huv_launch::probe_wait_ns();
      dim3 g(M / kTcBN, 2 * M / 128, nc);
      prof.begin("tc_dft_gemm<sumsq>", st);
      tc_dft_gemm<0><<<g, 192, smem_tc, st>>>(tc.map_ae, mbE, tc.map_ae, p);
      prof.end(st);
      check_cuda(cudaGetLastError(), "tc_dft_gemm<0>");
    }
    if (sep) {
      interp_separable(ds, M, nc, IM, mean, BI, o, st, true);
    } else {
      prof.begin("interp_band", st);
      check_cuda(band_forward(IM, HUV_INPUT_RASTER_F32, M, lgm, h2, nc, X2, C, nullptr, nullptr, nullptr, twm, st,
                              nullptr, nullptr),
                 "band_forward(interp)");
      prof.end(st);
      prof.begin("socs_rows_tc<interp>", st);
      const float scale = 1.0f / (static_cast<float>(M) * static_cast<float>(M));
      launch_rows(nullptr, scale, C, 1, h2, h2, nrI, n, kbI, 0, BI, twn, nc, st);
      check_cuda(cudaGetLastError(), "socs_rows_tc(interp)");
      prof.end(st);
    }
    if (!sep) {
      TcGemmParams p{};
      p.kboxes = kpI / 64;
      p.ksteps = kstI;
      p.G = n / kTcBN;
      p.a_rows = n;
      p.b_prob = 2 * n;
      p.b_step = kTcBN;
      p.b_plane = n;
      p.out_ld = n;
      p.out_plane = static_cast<long long>(n) * n;
      p.keep = 1.f;
      p.flare = 0.f;
      p.mean = nullptr;
      p.f16 = 0;
      p.out = o;
      p.err = dev_err;
      p.probe_wait_ns = huv_launch::probe_wait_ns();
      CUtensorMap mo;
      p.out_tma = make_out_map(&mo, o, static_cast<uint64_t>(nc) * n, n) ? 1 : 0;
      if (!p.out_tma) mo = tc.map_ai;  // unused
      dim3 g(1, n / 128, nc);
      CUtensorMap mbZ64;
      const int abox = (p.ksteps + 1) / 2;  // 32-wide A boxes
      const bool w256 = p.out_tma && n % 256 == 0 && abox <= 6 &&
                        make_map_sw64(&mbZ64, BI, static_cast<uint64_t>(nc) * 2 * n, kbI, 256, kcI, false);
      prof.begin("tc_dft_gemm<interp>", st);
      if (w256) {  // 128 x 256 tiles, A and B through 32-wide boxes
        p.G = n / 256;
        p.kboxes = abox;
        if (abox <= 5)
          tc_interp_w256<5, 7, 2><<<g, 192, w256_smem_bytes(5, 7, 2), st>>>(tc.map_ai32, mbZ64, mo, p);
        else
          tc_interp_w256<6, 6, 2><<<g, 192, w256_smem_bytes(6, 6, 2), st>>>(tc.map_ai32, mbZ64, mo, p);
      } else {
        tc_dft_gemm<1><<<g, 192, tc_smem_bytes(3, kTcBN, false, true), st>>>(tc.map_ai, mbI, mo, p);
      }
      prof.end(st);
      check_cuda(cudaGetLastError(), "tc_dft_gemm<1>");
    }
    // mask band (rows, columns, mean), 2 field launches (3 with the row GEMM), 2 (separable) or 4 interpolation launches
    // (the fused field pass is one launch, two when kernel groups are reduced)
    prof.launches += (sep ? 7 : (gemm_rows ? 10 : 9)) - (fused && field_fused_part_bytes(M, K) == 0 ? 1 : 0);
  }
}

bool Engine::separable_ok(const DeviceSet& ds, int M) const {
  return M <= 192 && M % 16 == 0 && M < n && huv_launch::xt_ok(M, ds.hb) && hybrid_supported(ds, M);
}

// P(Y, m) = (1/M) sum_{|f| <= h2} exp(2 pi i f (Y/N - m/M)) (a Dirichlet
// kernel) as FP16 hi/lo planes [2][N][192], built once per (set, M).
void Engine::interp_matrix(DeviceSet& ds, int M) {
  using namespace huv_launch;
  TcState& tc = ds.tc[M];
  const int h2 = 2 * ds.hb;
  if (!tc.gp) {
    constexpr int kpP = 192;
    std::vector<double> pm(static_cast<size_t>(n) * M);
    const double nm = static_cast<double>(n) * M;
    for (int y = 0; y < n; ++y)
      for (int m = 0; m < M; ++m) {
        // t = Y/N - m/M = q / (N M); sum_{|f|<=H} e^{2 pi i f t} = sin((2H+1) pi t) / sin(pi t)
        const long long q = static_cast<long long>(y) * M - static_cast<long long>(m) * n;
        const double v = q == 0 ? static_cast<double>(2 * h2 + 1)
                                : std::sin((2 * h2 + 1) * kPi * static_cast<double>(q) / nm) /
                                      std::sin(kPi * static_cast<double>(q) / nm);
        pm[static_cast<size_t>(y) * M + m] = v / M;
      }
    const auto pp = split_planes_f16(pm, n, M, kpP);
    check_cuda(cudaMalloc(&tc.gp, pp.size() * 2), "cudaMalloc(P)");
    check_cuda(cudaMemcpy(tc.gp, pp.data(), pp.size() * 2, cudaMemcpyHostToDevice), "upload P");
    if (!make_map(&tc.map_pi, tc.gp, 2ull * n, kpP, 128, 0, true) ||
        !make_map_sw64(&tc.map_pi32, tc.gp, 2ull * n, kpP, 128, kpP, true))
      throw Error(HUV_ERR_CUDA, "cuTensorMapEncodeTiled failed for the interpolation operand");
  }
}

void Engine::interp_separable(DeviceSet& ds, int M, int nc, const void* im_split, const float* mean, void* BIv,
                              float* o, cudaStream_t st, bool profile) {
  using namespace huv_launch;
  static std::atomic<uint64_t> smem_set{0};
  once_per_device(smem_set, [] { check_cuda(tc_set_smem(), "cudaFuncSetAttribute(tc)"); });
  interp_matrix(ds, M);
  TcState& tc = ds.tc[M];
  const void* IM = im_split;
  __nv_bfloat16* BI = static_cast<__nv_bfloat16*>(BIv);
  struct Region {  // the profiler's regions only when the caller is not inside one of its own
    Prof& pr;
    bool on;
    void begin(const char* nm, cudaStream_t s) {
      if (on) pr.begin(nm, s);
    }
    void end(cudaStream_t s) {
      if (on) pr.end(s);
    }
  } prof{this->prof, profile};
  CUtensorMap mbZ;
  {
    // Z^T[clip][plane][Y][y] = sum_x P(Y, x) I_M(y, x) / s, FP16 split planes:
    // A = P (rows Y), B = I_M / s (rows y, K = x), s = interp_scale(mean);
    // G1 clips per CTA share the A tile.  Each CTA takes half of the M
    // columns (N = M / 2), so that two clips' B tiles fit the ring
    // (tc_stages: 7 / 6 / 5 stages at M = 128 / 160 / 192).
    const int bn1 = M / 2;
    const int ntile1 = M / bn1, mtiles = n / 128;
    // Clips per CTA: the fewest (up to 32) whose grid fits one wave of one
    // CTA per SM, else 32.  Each CTA's run is latency-bound (how much of the
    // clips' B tiles is in flight), so longer runs over a resident A tile
    // beat more CTAs: at 128 clips 1 / 2 / 4 / 8 clips per CTA time
    // 1.24 / 1.12 / 1.03 / 0.99 ms per 20 launches (N = M); at 256 clips
    // and N = M, 15 per CTA (one wave of 144 CTAs) 0.084 ms per launch
    // against 0.092 with 8 (256 CTAs, 1.7 waves).
    int sms = 0, dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    int G1 = 32;
    for (int gc = 1; gc < 32; ++gc)
      if (static_cast<long long>(ntile1) * mtiles * ((nc + gc - 1) / gc) <= sms) {
        G1 = gc;
        break;
      }
    CUtensorMap mbS;
    if (!make_map(&mbS, IM, static_cast<uint64_t>(nc) * 2 * M, M, bn1, M, true) ||
        !make_map(&mbZ, BI, static_cast<uint64_t>(nc) * 2 * n, M, kTcBN, M, true))
      throw Error(HUV_ERR_CUDA, "cuTensorMapEncodeTiled failed for the interpolation operands");
    TcGemmParams p{};
    p.kboxes = (M + 63) / 64;
    p.ksteps = M / 16;
    p.G = G1;
    p.nprob = nc;
    p.a_rows = n;
    p.b_prob = G1 * 2 * M;
    p.b_step = 2 * M;
    p.b_plane = M;
    p.err = dev_err;
    p.probe_wait_ns = huv_launch::probe_wait_ns();
    p.bop = BI;
    p.bop_prob = 2ll * n * M;
    p.bop_plane = static_cast<long long>(n) * M;
    p.bop_ld = M;
    const dim3 g(ntile1, mtiles, (nc + G1 - 1) / G1);
    prof.begin("tc_dft_gemm<interp_x>", st);
    if (bn1 == 64)
      tc_dft_gemm<3, 64><<<g, 192, tc_smem_bytes(p.kboxes, 64, false, false, tc_stages(3, 64)), st>>>(
          tc.map_pi, mbS, tc.map_pi, p);
    else if (bn1 == 80)
      tc_dft_gemm<3, 80><<<g, 192, tc_smem_bytes(p.kboxes, 80, false, false, tc_stages(3, 80)), st>>>(
          tc.map_pi, mbS, tc.map_pi, p);
    else if (bn1 == 96)
      tc_dft_gemm<3, 96><<<g, 192, tc_smem_bytes(p.kboxes, 96, false, false, tc_stages(3, 96)), st>>>(
          tc.map_pi, mbS, tc.map_pi, p);
    else
      throw Error(HUV_ERR_UNSUPPORTED, "separable interpolation: evaluation grid must be 128, 160 or 192");
    prof.end(st);
    check_cuda(cudaGetLastError(), "tc_dft_gemm<3>");
  }
  TcGemmParams p{};
  p.kboxes = (M + 63) / 64;
  p.ksteps = M / 16;
  p.G = n / kTcBN;
  p.a_rows = n;
  p.b_prob = 2 * n;
  p.b_step = kTcBN;
  p.b_plane = n;
  p.out_ld = n;
  p.out_plane = static_cast<long long>(n) * n;
  p.keep = 1.f;
  p.flare = 0.f;
  p.mean = mean;  // undo the planes' scale
  p.f16 = 1;
  p.out = o;
  p.err = dev_err;
  p.probe_wait_ns = huv_launch::probe_wait_ns();
  CUtensorMap mo;
  p.out_tma = make_out_map(&mo, o, static_cast<uint64_t>(nc) * n, n) ? 1 : 0;
  if (!p.out_tma) mo = tc.map_pi;  // unused
  dim3 g(1, n / 128, nc);
  CUtensorMap mbZ64;
  const int abox = (p.ksteps + 1) / 2;  // 32-wide A boxes
  const bool w256 = p.out_tma && n % 256 == 0 && abox <= 6 &&
                    make_map_sw64(&mbZ64, BI, static_cast<uint64_t>(nc) * 2 * n, M, 256, M, true);
  prof.begin("tc_dft_gemm<interp>", st);
  if (w256) {  // 128 x 256 tiles, A and B through 32-wide boxes
    p.G = n / 256;
    p.kboxes = abox;
    if (abox <= 5)
      tc_interp_w256<5, 7, 2><<<g, 192, w256_smem_bytes(5, 7, 2), st>>>(tc.map_pi32, mbZ64, mo, p);
    else
      tc_interp_w256<6, 6, 2><<<g, 192, w256_smem_bytes(6, 6, 2), st>>>(tc.map_pi32, mbZ64, mo, p);
  } else {
    tc_dft_gemm<1><<<g, 192, tc_smem_bytes(3, kTcBN, false, true), st>>>(tc.map_pi, mbZ, mo, p);
  }
  prof.end(st);
  check_cuda(cudaGetLastError(), "tc_dft_gemm<1>");
}
}  // namespace huv

extern "C" huv_status huv_debug_probe_wait(int64_t ns) {
  huv_launch::g_probe_wait_ns.store(ns > 0 ? static_cast<unsigned long long>(ns) : 0ull);
  return HUV_OK;
}
