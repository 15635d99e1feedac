// Row band of 8-bit mask rasters on the tensor cores (tcgen05.mma kind::i8,
// sm_100a): the first half of Mask::spectrum's raster path
// (crates/highuvlith-core/src/mask.rs:630-635) restricted to the orders
// |m| <= hb that the SOCS kernels keep.
//
//   X(y, m) = sum_x mask(y, x) e^{-2 pi i m x / L}
//
// is a GEMM of the mask rows (u8, exact) against a quantised twiddle matrix.
// Its columns n are one column of ones (n = 0), cos(2 pi m x / L) for
// m = 0..hb (n = 1 + m) and sin(2 pi m x / L) for m = 1..hb (n = hb + 1 + m).
// Each twiddle value t is stored as the integer
//     T = round(t 2^20) + 2^20  in [0, 2^21]
// split into three unsigned base-256 digit planes, so that three u8 x u8
// MMAs give exact s32 sums (255 * 255 * L < 2^31 for L <= 2^15) and
//     sum_x mask t = (2^16 acc0 + 2^8 acc1 + acc2 - 2^20 rowsum) / 2^20
// exactly in 64-bit integers, rowsum being the ones column.  The only error
// is the twiddle quantisation (|dt| <= 2^-21 per term), below the FP32
// rounding of a radix-4 FFT of the same row.  The input is real, so orders
// m < 0 are the conjugates of m > 0.
//
// Roles per CTA (6 warps, 128 mask rows): warp 0 issues TMA loads (no
// multicast) of 128 x 128 mask tiles and the three N x 128 digit tiles per
// K box, warp 1 issues the MMAs from one thread into three accumulators in
// tensor memory, warps 2-5 combine the digits, stage the rows in shared
// memory and write X[row][m + hb] (float2) with coalesced stores.  Every
// mbarrier wait is bounded in time; a timeout sets the error flag, drains
// in-flight work with bounded waits, frees tensor memory and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <vector>

#include "tc_ptx.cuh"

namespace huv_dev {

constexpr int kMbStages = 2;
constexpr uint32_t kMbABox = 128 * 128;  // 128 rows x 128 u8
constexpr uint64_t kMbWaitNs = 2000000000ull;
constexpr int kMbTwShift = 20;  // twiddles quantised to 2^-20

__host__ __device__ constexpr uint32_t mb_stage_bytes(int N) { return kMbABox + 3u * static_cast<uint32_t>(N) * 128u; }
__host__ __device__ constexpr size_t mb_smem_bytes(int N) {
  return 1024 + kMbStages * static_cast<size_t>(mb_stage_bytes(N)) + 256;
}

// grid: (rows / 128); rows = clips * L.  X: [rows][2 hb + 1], or with
// `transposed` the orders m = 0..hb alone as [clip][hb + 1][L] (each
// order's column contiguous in y; the orders m < 0 are their conjugates).
__global__ void __launch_bounds__(192, 1)
    band_rows_i8(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmD, int kboxes,
                 int N, int hb, uint32_t tmem_cols, int L, int transposed, float2* __restrict__ X, int* err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t stage_bytes = mb_stage_bytes(N);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kMbStages * stage_bytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + kMbStages;
  uint64_t* tfull = bars + 2 * kMbStages;
  uint64_t* done = bars + 2 * kMbStages + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kMbStages + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kMbStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tfull, 1);
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  auto fail = [&](int code) {
    *abort_flag = 1;
    if (err) atomicExch(err, code);
  };

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&tmA);
      prefetch_tmap(&tmD);
      int kb = 0;
      for (; kb < kboxes && !*abort_flag; ++kb) {
        const int s = kb % kMbStages;
        if (!mbar_wait(&empty[s], ((kb / kMbStages) & 1) ^ 1, kMbWaitNs)) {
          fail(11);
          break;
        }
        uint8_t* st = base + s * stage_bytes;
        mbar_arrive_expect_tx(&full[s], stage_bytes);
        tma_load_2d(st, &tmA, kb * 128, row0, &full[s]);
        for (int d = 0; d < 3; ++d) tma_load_2d(st + kMbABox + d * N * 128, &tmD, kb * 128, d * N, &full[s]);
      }
      // Drain: every load issued must have landed before the CTA may exit.
      for (int q = (kb > kMbStages ? kb - kMbStages : 0); q < kb; ++q)
        mbar_wait(&full[q % kMbStages], (q / kMbStages) & 1, kMbWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_u8(128, N);
      bool ok = true;
      for (int kb = 0; kb < kboxes && !*abort_flag; ++kb) {
        const int s = kb % kMbStages;
        if (!mbar_wait(&full[s], (kb / kMbStages) & 1, kMbWaitNs)) {
          fail(12);
          ok = false;
          break;
        }
        tc_fence_after();
        uint8_t* st = base + s * stage_bytes;
        const uint64_t a = smem_desc_sw128(smem_u32(st));
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t adv = static_cast<uint64_t>(2 * ks);  // 32 bytes per 32-wide K step
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const uint64_t b = smem_desc_sw128(smem_u32(st + kMbABox + d * N * 128));
            tc_mma_i8(tmem_base + d * N, a + adv, b + adv, idesc, (kb | ks) ? 1u : 0u);
          }
        }
        tc_commit(&empty[s]);
      }
      if (ok && !*abort_flag) tc_commit(tfull);
      // All MMAs issued by this thread have completed once `done` flips.
      tc_commit(done);
      mbar_wait(done, 0, kMbWaitNs);
    }
  } else {
    // Epilogue warps 2..5: TMEM lane quadrant = warp % 4, one mask row per thread.
    const int quad = warp & 3;
    const bool got = __all_sync(0xffffffffu, mbar_wait(tfull, 0, kMbWaitNs));
    if (!got) {
      if (lane == 0) fail(13);
    } else {
      tc_fence_after();
      // The stage buffers are free: every MMA that read them has completed.
      const int ld = N + 1;
      float* stage = reinterpret_cast<float*>(base) + quad * 32 * ld;
      const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quad * 32) << 16);
      long long rowsum = 0;
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v0[16], v1[16], v2[16];
        tmem_ld16(taddr + c0, v0);
        tmem_ld16(taddr + N + c0, v1);
        tmem_ld16(taddr + 2 * N + c0, v2);
        if (c0 == 0) rowsum = __float_as_int(v2[0]);  // ones column: digits (0, 0, 1)
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const long long t = (static_cast<long long>(__float_as_int(v0[i])) << 16) +
                              (static_cast<long long>(__float_as_int(v1[i])) << 8) +
                              static_cast<long long>(__float_as_int(v2[i])) - (rowsum << kMbTwShift);
          stage[lane * ld + c0 + i] = static_cast<float>(t) * (1.0f / static_cast<float>(1 << kMbTwShift));
        }
      }
      __syncwarp();
      const int B = 2 * hb + 1;
      if (transposed) {
        // orders m = 0..hb only (the raster is real, X(y, -m) = conj X(y, m)),
        // one order per store: 32 consecutive y of one column (256 bytes)
        const int grow = row0 + quad * 32;
        const int clip = grow / L, y0 = grow - clip * L;
        float2* out = X + static_cast<size_t>(clip) * (hb + 1) * L + y0 + lane;
        for (int m = 0; m <= hb; ++m) {
          const float c = stage[lane * ld + 1 + m];
          const float s = m ? stage[lane * ld + hb + 1 + m] : 0.f;
          out[static_cast<size_t>(m) * L] = make_float2(c, -s);
        }
      } else {
        float2* out = X + static_cast<size_t>(row0 + quad * 32) * B;
        for (int w = lane; w < 32 * B; w += 32) {
          const int r = w / B, mi = w - r * B;
          const int m = mi - hb, am = m < 0 ? -m : m;
          const float c = stage[r * ld + 1 + am];
          const float s = am ? stage[r * ld + hb + 1 + am] : 0.f;
          out[w] = make_float2(c, m >= 0 ? -s : s);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, tmem_cols);
}

}  // namespace huv_dev

// ------------------------------------------------------------------ host
namespace huv_launch {

using namespace huv_dev;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_u8_fn() {
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

// 2-D u8 tensor map over [rows][cols] (row stride cols bytes), box 128 x box_rows, 128B swizzle.
bool make_u8_map(CUtensorMap* map, const void* ptr, uint64_t rows, uint64_t cols, int box_rows) {
  auto fn = encode_u8_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols)};
  cuuint32_t box[2] = {128, static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Columns of the digit planes for band half-width hb: ones + (hb + 1) cos +
// hb sin, rounded up to a multiple of 16 (the MMA's N granularity).
int mask_rows_tc_cols(int hb) { return (2 * hb + 2 + 15) / 16 * 16; }

// Whether the tensor-core row band applies: rows a multiple of 128, three
// accumulators within the 512 tensor-memory columns, exact s32 sums, and a
// driver entry point for tensor maps.
bool mask_rows_tc_supported(int n, int hb) {
  return n >= 128 && n % 128 == 0 && n <= 32768 && 3 * mask_rows_tc_cols(hb) <= 512 && encode_u8_fn() != nullptr;
}

// Digit planes [3][N][n] (u8) of the quantised twiddle matrix, built in FP64
// with exact argument reduction (m x mod n).
std::vector<uint8_t> mask_rows_tc_digits(int n, int hb) {
  const int N = mask_rows_tc_cols(hb);
  std::vector<uint8_t> tab(3 * static_cast<size_t>(N) * n, 0);
  const double two_pi = 6.283185307179586476925286766559;
  const double q = static_cast<double>(1 << kMbTwShift);
  for (int c = 0; c < 2 * hb + 2; ++c)
    for (int x = 0; x < n; ++x) {
      long long T;
      if (c == 0) {
        T = 1;  // the ones column, read back as the row sum
      } else {
        const bool is_cos = c <= hb + 1;
        const long long m = is_cos ? c - 1 : c - hb - 1;
        const double th = two_pi * static_cast<double>((m * x) % n) / n;
        T = std::llround((is_cos ? std::cos(th) : std::sin(th)) * q) + (1ll << kMbTwShift);
      }
      tab[(0 * static_cast<size_t>(N) + c) * n + x] = static_cast<uint8_t>(T >> 16);
      tab[(1 * static_cast<size_t>(N) + c) * n + x] = static_cast<uint8_t>((T >> 8) & 255);
      tab[(2 * static_cast<size_t>(N) + c) * n + x] = static_cast<uint8_t>(T & 255);
    }
  return tab;
}

// X[clip][y][m + hb] (or, with `transposed`, X[clip][m][y] for m = 0..hb) for u8
// rasters [clips][n][n] on the tensor cores.  `digits` is
// mask_rows_tc_digits(n, hb) on the device.  Returns cudaErrorNotSupported
// when the shape or the input's alignment rules the path out (the caller
// then takes the FFT path).
cudaError_t mask_rows_tc(const void* in, int n, int hb, int clips, float2* X, const uint8_t* digits, int* err,
                         cudaStream_t st, bool transposed) {
  if (!digits || !mask_rows_tc_supported(n, hb) || (reinterpret_cast<uintptr_t>(in) & 15u) != 0)
    return cudaErrorNotSupported;
  const int N = mask_rows_tc_cols(hb);
  // the attribute is per device: bit d set once device d has it
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return e;
  const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t(1) << dev) : 0;
  if (!bit || !(attr_set.load(std::memory_order_acquire) & bit)) {
    cudaError_t e = cudaFuncSetAttribute(band_rows_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(mb_smem_bytes(160) + (40 << 10)));
    if (e != cudaSuccess) return e;
    if (bit) attr_set.fetch_or(bit, std::memory_order_acq_rel);
  }
  CUtensorMap ma, md;
  if (!make_u8_map(&ma, in, static_cast<uint64_t>(clips) * n, n, 128) ||
      !make_u8_map(&md, digits, 3ull * N, n, N))
    return cudaErrorNotSupported;
  // Two CTAs share an SM when both fit in shared memory and tensor memory
  // (256 columns each); with 512 columns the request is padded so that one
  // CTA holds the SM and no allocation waits on another CTA.
  const uint32_t cols = 3 * N <= 256 ? 256u : 512u;
  size_t smem = mb_smem_bytes(N);
  if (cols == 512u && smem < (120u << 10)) smem = 120u << 10;
  band_rows_i8<<<clips * n / 128, 192, smem, st>>>(ma, md, n / 128, N, hb, cols, n, transposed ? 1 : 0, X, err);
  return cudaGetLastError();
}

}  // namespace huv_launch
