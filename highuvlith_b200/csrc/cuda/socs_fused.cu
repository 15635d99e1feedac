// Fused field pass of the SOCS sum on the evaluation grid (L = 128, 160).
//
// One CTA of 512 threads takes one clip and a group of G kernels.  For each
// kernel k of the group it forms the band products P = kappa_k . M (B x B,
// B = 2 h + 1) round by round, transforms the band rows along x into
// T[x][my] (L x B complex, held in shared memory, never in HBM), then
// transforms every column x of T along y and adds |E_k|^2 into registers:
// the same inverse transforms as the reference's row-pruned 2-D IFFT per
// kernel (fft2d.rs:166-170, aerial.rs:1682-1721), on the coarse grid.
//
// Transforms are two register-radix Stockham passes (fft_reg.cuh): a
// radix-16 first pass over the zero-padded band and a last pass of radix
// Q = L / 16 (8, 10, 12).  Sequences are processed 32 at a time; lane
// s = t % 32 owns sequence s of the round and j = t / 32 is its butterfly, so
// the last pass of every round gives a thread the outputs x (or y) = j + 16 p
// of one sequence: its twiddles are the same in every pass and its column
// outputs land in fixed accumulator registers across kernels.
//
// Shared memory (float2): T [L][B] (ld = B, odd, so the column pass's
// strided reads are conflict-free), C [L][32] (the rounds' intermediate,
// sequence-minor), P [32][B] (the round's band products).  A thread holds
// (L / 32) Q accumulators: 32 at L = 128, 50 at L = 160 (128 registers, no
// spills); L = 192 would need 72 and spills, so it keeps the two-kernel pass.
//
// Output: with one group per clip the CTA applies the normalisation and
// flare epilogue itself, out = keep * sum + flare * mean (FP32 [clip][L][L],
// or v = out / interp_scale(mean) as FP16 hi/lo planes [clip][2][L][L] for
// the separable tensor-core interpolation); with several groups it writes
// its partial sum to part[clip][group][L][L] and field_reduce adds the groups
// in index order (deterministic) and applies the epilogue.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fft_reg.cuh"

namespace huv_dev {

constexpr int kFusedThreads = 512;
constexpr int kFusedRound = 32;      // sequences per round
constexpr int kFusedGroup = 8;       // kernels per CTA

__host__ __device__ constexpr size_t fused_smem_bytes(int L, int B) {
  return (static_cast<size_t>(L) * B + static_cast<size_t>(L) * kFusedRound +
          static_cast<size_t>(kFusedRound) * B) * sizeof(float2);
}

__device__ __forceinline__ float2 fused_cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Band position of zero-padded element i of an L-point sequence: the order
// o = i (i <= h) or i - L (i >= L - h), stored at column o + h; -1 outside.
__device__ __forceinline__ int band_col(int i, int L, int hb) {
  return i <= hb ? i + hb : (i >= L - hb ? i - L + hb : -1);
}

template <int L>
__global__ void __launch_bounds__(kFusedThreads, 1)
    field_fused_kernel(const float2* __restrict__ kband, const float2* __restrict__ Mband, int K, int hb, int groups,
                     float keep, float flare, const float* __restrict__ mean, float* __restrict__ out,
                     __half* __restrict__ split, float* __restrict__ part, const float2* __restrict__ tw) {
  constexpr int Q = L / 16;            // radix of the last pass
  constexpr int CR = L / kFusedRound;  // column rounds
  extern __shared__ float2 sm[];
  const int B = 2 * hb + 1;
  float2* T = sm;                                       // [L][B]
  float2* C = T + static_cast<size_t>(L) * B;           // [L][32]
  float2* P = C + static_cast<size_t>(L) * kFusedRound;  // [32][B]
  const int t = threadIdx.x;
  const int s = t & 31, j = t >> 5;  // lane: sequence of the round; warp: butterfly
  const int clip = blockIdx.y, grp = blockIdx.x;
  const int k0 = grp * kFusedGroup, k1 = min(K, k0 + kFusedGroup);
  const float2* Mc = Mband + static_cast<size_t>(clip) * B * B;

  // last-pass twiddles w^{r j}, r = 1 .. Q - 1, inverse direction (the same
  // for the row and the column passes: both have butterfly j = t / 32)
  float2 w[Q - 1];
#pragma unroll
  for (int r = 1; r < Q; ++r) {
    const float2 x = tw[r * j];
    w[r - 1] = make_float2(x.x, -x.y);
  }
  float acc[CR][Q];
#pragma unroll
  for (int c = 0; c < CR; ++c)
#pragma unroll
    for (int p = 0; p < Q; ++p) acc[c][p] = 0.f;

  const bool first = t < kFusedRound * Q;  // first-pass butterflies: Q per sequence
  const int jf = t >> 5;                    // first-pass butterfly of this thread (t < 32 Q)

  for (int k = k0; k < k1; ++k) {
    const float2* Kk = kband + static_cast<size_t>(k) * B * B;
    // ---------------- rows: band rows my0 .. my0 + 31 along x -> T[x][my]
    for (int my0 = 0; my0 < B; my0 += kFusedRound) {
      const int nseq = min(kFusedRound, B - my0);
      // P[q][mx] = kappa_k[my0 + q][mx] M[my0 + q][mx] (zero past the band)
      for (int e = t; e < kFusedRound * B; e += kFusedThreads) {
        const int q = e / B;
        float2 v = make_float2(0.f, 0.f);
        if (q < nseq) {
          const size_t o = static_cast<size_t>(my0) * B + e;
          v = fused_cmul(Kk[o], Mc[o]);
        }
        P[e] = v;
      }
      __syncthreads();
      if (first) {
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int mx = band_col(jf + r * Q, L, hb);
          v[r] = mx >= 0 ? P[s * B + mx] : make_float2(0.f, 0.f);
        }
        fr_dft<16, +1>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) C[(jf * 16 + r) * kFusedRound + s] = v[r];
      }
      __syncthreads();
      {
        float2 v[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) v[r] = C[(j + 16 * r) * kFusedRound + s];
#pragma unroll
        for (int r = 1; r < Q; ++r) v[r] = fused_cmul(v[r], w[r - 1]);
        fr_dft<Q, +1>(v);
        if (s < nseq) {
#pragma unroll
          for (int p = 0; p < Q; ++p) T[static_cast<size_t>(j + 16 * p) * B + my0 + s] = v[p];
        }
      }
      // the next round's P and C writes come after its own first barrier
    }
    __syncthreads();  // T complete
    // ---------------- columns: x0 .. x0 + 31 along y, |E|^2 into registers
#pragma unroll
    for (int c = 0; c < CR; ++c) {
      const int x = c * kFusedRound + s;
      if (first) {
        float2 v[16];
        const float2* col = T + static_cast<size_t>(x) * B;
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int my = band_col(jf + r * Q, L, hb);
          v[r] = my >= 0 ? col[my] : make_float2(0.f, 0.f);
        }
        fr_dft<16, +1>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) C[(jf * 16 + r) * kFusedRound + s] = v[r];
      }
      __syncthreads();
      {
        float2 v[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) v[r] = C[(j + 16 * r) * kFusedRound + s];
#pragma unroll
        for (int r = 1; r < Q; ++r) v[r] = fused_cmul(v[r], w[r - 1]);
        fr_dft<Q, +1>(v);
#pragma unroll
        for (int p = 0; p < Q; ++p) acc[c][p] += v[p].x * v[p].x + v[p].y * v[p].y;
      }
      __syncthreads();  // C is rewritten by the next round (or the next kernel's rows)
    }
  }

  // ---------------- output: thread (c, p) holds pixel (y = j + 16 p, x = 32 c + s)
  if (groups > 1) {
    float* pc = part + (static_cast<size_t>(clip) * groups + grp) * L * L;
#pragma unroll
    for (int c = 0; c < CR; ++c)
#pragma unroll
      for (int p = 0; p < Q; ++p) pc[static_cast<size_t>(j + 16 * p) * L + c * kFusedRound + s] = acc[c][p];
    return;
  }
  const float add = mean ? flare * mean[clip] : 0.f;
  const float inv = split ? 1.f / interp_scale(mean ? mean[clip] : 0.f) : 1.f;
#pragma unroll
  for (int c = 0; c < CR; ++c)
#pragma unroll
    for (int p = 0; p < Q; ++p) {
      const size_t o = static_cast<size_t>(j + 16 * p) * L + c * kFusedRound + s;
      const float v = keep * acc[c][p] + add;
      if (split) {
        const float sv = v * inv;
        const __half hi = __float2half_rn(sv);
        __half* sc = split + static_cast<size_t>(clip) * 2 * L * L + o;
        sc[0] = hi;
        sc[static_cast<size_t>(L) * L] = __float2half_rn(sv - __half2float(hi));
      } else {
        out[static_cast<size_t>(clip) * L * L + o] = v;
      }
    }
}

// Sum of the groups' partials (in group order) with the epilogue of
// socs_field_fused.  grid: (ceil(L^2 / 256), clips).
__global__ void field_reduce(const float* __restrict__ part, int groups, int L, float keep, float flare,
                             const float* __restrict__ mean, float* __restrict__ out, __half* __restrict__ split) {
  const int clip = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int LL = L * L;
  if (i >= LL) return;
  const float* pc = part + static_cast<size_t>(clip) * groups * LL + i;
  float a = 0.f;
  for (int g = 0; g < groups; ++g) a += pc[static_cast<size_t>(g) * LL];
  const float v = keep * a + (mean ? flare * mean[clip] : 0.f);
  if (split) {
    const float sv = v / interp_scale(mean ? mean[clip] : 0.f);
    const __half hi = __float2half_rn(sv);
    __half* sc = split + static_cast<size_t>(clip) * 2 * LL + i;
    sc[0] = hi;
    sc[LL] = __float2half_rn(sv - __half2float(hi));
  } else {
    out[static_cast<size_t>(clip) * LL + i] = v;
  }
}

}  // namespace huv_dev

namespace huv_launch {

using namespace huv_dev;

// Whether the fused field pass serves an L-point grid with band half-width
// hb (its shared memory must fit one CTA).
bool field_fused_ok(int L, int hb) {
  if (!(L == 128 || L == 160) || 2 * hb >= L) return false;
  return fused_smem_bytes(L, 2 * hb + 1) <= 227 * 1024;
}

// Kernel groups per clip of the fused field pass, and the partial-sum bytes
// per clip it needs (0 with one group).
int field_fused_groups(int K) { return (K + kFusedGroup - 1) / kFusedGroup; }
size_t field_fused_part_bytes(int L, int K) {
  const int g = field_fused_groups(K);
  return g > 1 ? static_cast<size_t>(g) * L * L * sizeof(float) : 0;
}

// The field pass of `clips` clips: out (FP32 [clip][L][L]) or, with split
// set, FP16 hi/lo planes of out / interp_scale(mean).  `part` needs
// clips * field_fused_part_bytes(L, K) bytes when K > 8.
cudaError_t socs_field_fused(const float2* kband, const float2* Mband, int K, int hb, int L, int clips, float keep,
                             float flare, const float* mean, float* out, void* split, float* part, const float2* tw,
                             cudaStream_t st) {
  if (!field_fused_ok(L, hb) || K < 1 || (split && !mean)) return cudaErrorInvalidValue;
  const int groups = field_fused_groups(K);
  if (groups > 1 && !part) return cudaErrorInvalidValue;
  const size_t sm = fused_smem_bytes(L, 2 * hb + 1);
  __half* sp = static_cast<__half*>(split);
  const dim3 g(groups, clips);
  switch (L) {
    case 128:
      field_fused_kernel<128><<<g, kFusedThreads, sm, st>>>(kband, Mband, K, hb, groups, keep, flare, mean, out, sp,
                                                           part, tw);
      break;
    default:
      field_fused_kernel<160><<<g, kFusedThreads, sm, st>>>(kband, Mband, K, hb, groups, keep, flare, mean, out, sp,
                                                             part, tw);
      break;
  }
  if (groups > 1) {
    const dim3 gr((L * L + 255) / 256, clips);
    field_reduce<<<gr, 256, 0, st>>>(part, groups, L, keep, flare, mean, out, sp);
  }
  return cudaGetLastError();
}

cudaError_t field_fused_set_smem() {
  cudaError_t e = cudaFuncSetAttribute(field_fused_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(field_fused_kernel<160>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return e;
}

}  // namespace huv_launch
