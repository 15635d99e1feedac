// Fused field pass of the SOCS sum on the evaluation grid (L = 128, 160).
//
// One CTA of 512 threads (16 warps) takes one clip and a group of G kernels.
// For each kernel k of the group it transforms the band rows of the
// products P = kappa_k . M (B x B, B = 2 h + 1) along x into T[x][my]
// (L x B complex, held in shared memory, never in HBM), then transforms
// every column x of T along y and adds |E_k|^2 into registers: the same
// inverse transforms as the reference's row-pruned 2-D IFFT per kernel
// (fft2d.rs:166-170, aerial.rs:1682-1721), on the coarse grid.
//
// Each warp transforms two sequences at a time on its own, with only warp
// barriers: the rows in pairs (my, my + 1) handed out round-robin over the
// warps, then the columns in pairs (x, x + 1), five (L = 160) or four
// (L = 128) per warp.  The CTA synchronises twice per kernel (rows done,
// columns done), so a warp's loads and shared-memory round trips overlap
// the other warps' arithmetic.  Transforms are two register-radix Stockham
// passes (fft_reg.cuh): a radix-16 first pass over the zero-padded band
// (lanes (c, jf), c = lane / Q, jf = lane % Q: 2 Q lanes) and a last pass of
// radix Q = L / 16 (lanes (c, j), c = lane / 16, j = lane % 16: all 32).  A
// lane's last-pass butterfly j is the same in every pass, so its twiddles are
// loaded once and its column outputs (y = j + 16 p) land in fixed
// accumulator registers across kernels: (L / 32) Q of them, 50 at L = 160
// (128 registers, no spills); L = 192 would need 72 and keeps the two-kernel
// pass.
//
// Shared memory (float2): T [L][B] (ld = B, odd: the column pass's strided
// reads are conflict-free), the clip's mask band M [B][B], and per warp an
// intermediate C [2][L + L / 16] (element i of sequence c at
// c (L + L / 16) + i + i / 16: conflict-free first-pass stores and last-pass
// loads).  At the end the accumulators are staged through shared memory and
// written as coalesced rows.
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
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kFusedGroup = 8;  // kernels per CTA

__host__ __device__ constexpr int fused_lp(int L) { return L + L / 16; }
// T, M and the warps' intermediates; at least the L x L floats the output
// is staged through at the end (more than the rest when the band is narrow)
__host__ __device__ constexpr size_t fused_smem_bytes(int L, int B) {
  return (static_cast<size_t>(L) * B + static_cast<size_t>(B) * B +
          static_cast<size_t>(kFusedWarps) * 2 * fused_lp(L)) * sizeof(float2) >
                 static_cast<size_t>(L) * L * sizeof(float)
             ? (static_cast<size_t>(L) * B + static_cast<size_t>(B) * B +
                static_cast<size_t>(kFusedWarps) * 2 * fused_lp(L)) * sizeof(float2)
             : static_cast<size_t>(L) * L * sizeof(float);
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
  constexpr int Q = L / 16;       // radix of the last pass
  constexpr int LP = fused_lp(L);  // padded intermediate sequence length
  constexpr int CP = L / 32;      // column pairs per warp
  extern __shared__ float2 sm[];
  const int B = 2 * hb + 1;
  float2* T = sm;                                  // [L][B]
  float2* Ms = T + static_cast<size_t>(L) * B;     // [B][B]
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  float2* Cw = Ms + static_cast<size_t>(B) * B + warp * 2 * LP;  // this warp's [2][LP]
  const int clip = blockIdx.y, grp = blockIdx.x;
  const int k0 = grp * kFusedGroup, k1 = min(K, k0 + kFusedGroup);

  // the clip's mask band, once
  const float2* Mc = Mband + static_cast<size_t>(clip) * B * B;
  for (int e = t; e < B * B; e += kFusedThreads) Ms[e] = Mc[e];

  // first-pass lane roles: sequence c1 of the pair, butterfly jf (2 Q lanes)
  const bool fp = lane < 2 * Q;
  const int c1 = lane / Q, jf = lane - (lane / Q) * Q;
  // last-pass lane roles: sequence c2, butterfly j; twiddles w^{r j}, inverse
  const int c2 = lane >> 4, j = lane & 15;
  float2 w[Q - 1];
#pragma unroll
  for (int r = 1; r < Q; ++r) {
    const float2 x = tw[r * j];
    w[r - 1] = make_float2(x.x, -x.y);
  }
  float acc[CP][Q];
#pragma unroll
  for (int q = 0; q < CP; ++q)
#pragma unroll
    for (int p = 0; p < Q; ++p) acc[q][p] = 0.f;
  __syncthreads();

  for (int k = k0; k < k1; ++k) {
    const float2* Kk = kband + static_cast<size_t>(k) * B * B;
    // ---------------- rows: pairs (my, my + 1) along x -> T[x][my]
    for (int pr = warp; 2 * pr < B; pr += kFusedWarps) {
      if (fp) {
        const int my = 2 * pr + c1;
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (r >= 4 && r < 12) continue;  // outside the band (h < L / 4)
          const int mx = band_col(jf + r * Q, L, hb);
          v[r] = (mx >= 0 && my < B) ? fused_cmul(Kk[my * B + mx], Ms[my * B + mx]) : make_float2(0.f, 0.f);
        }
        fr_dft16_band<+1>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) Cw[c1 * LP + jf * 17 + r] = v[r];
      }
      __syncwarp();
      {
        float2 v[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) v[r] = Cw[c2 * LP + j + 17 * r];
#pragma unroll
        for (int r = 1; r < Q; ++r) v[r] = fused_cmul(v[r], w[r - 1]);
        fr_dft<Q, +1>(v);
        const int my = 2 * pr + c2;
        if (my < B) {
#pragma unroll
          for (int p = 0; p < Q; ++p) T[static_cast<size_t>(j + 16 * p) * B + my] = v[p];
        }
      }
      __syncwarp();
    }
    __syncthreads();  // T complete
    // ---------------- columns: pairs (x, x + 1) along y, |E|^2 into registers
#pragma unroll
    for (int q = 0; q < CP; ++q) {
      const int x0 = 2 * (warp + kFusedWarps * q);
      if (fp) {
        const float2* col = T + static_cast<size_t>(x0 + c1) * B;
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (r >= 4 && r < 12) continue;  // outside the band (h < L / 4)
          const int my = band_col(jf + r * Q, L, hb);
          v[r] = my >= 0 ? col[my] : make_float2(0.f, 0.f);
        }
        fr_dft16_band<+1>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) Cw[c1 * LP + jf * 17 + r] = v[r];
      }
      __syncwarp();
      {
        float2 v[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) v[r] = Cw[c2 * LP + j + 17 * r];
#pragma unroll
        for (int r = 1; r < Q; ++r) v[r] = fused_cmul(v[r], w[r - 1]);
        fr_dft<Q, +1>(v);
#pragma unroll
        for (int p = 0; p < Q; ++p) acc[q][p] += v[p].x * v[p].x + v[p].y * v[p].y;
      }
      __syncwarp();
    }
    __syncthreads();  // the next kernel's rows overwrite T
  }

  // ---------------- output: lane (q, p) holds pixel (y = j + 16 p, x = 2 (warp + 16 q) + c2);
  // staged as [y][x] floats over the (now free) shared memory, then coalesced rows
  float* S = reinterpret_cast<float*>(sm);
#pragma unroll
  for (int q = 0; q < CP; ++q)
#pragma unroll
    for (int p = 0; p < Q; ++p) S[(j + 16 * p) * L + 2 * (warp + kFusedWarps * q) + c2] = acc[q][p];
  __syncthreads();
  if (groups > 1) {
    float* pc = part + (static_cast<size_t>(clip) * groups + grp) * L * L;
    for (int e = t; e < L * L / 4; e += kFusedThreads)
      reinterpret_cast<float4*>(pc)[e] = reinterpret_cast<const float4*>(S)[e];
    return;
  }
  const float add = mean ? flare * mean[clip] : 0.f;
  const float inv = split ? 1.f / interp_scale(mean ? mean[clip] : 0.f) : 1.f;
  for (int e = t; e < L * L; e += kFusedThreads) {
    const float v = keep * S[e] + add;
    if (split) {
      const float sv = v * inv;
      const __half hi = __float2half_rn(sv);
      __half* sc = split + static_cast<size_t>(clip) * 2 * L * L + e;
      sc[0] = hi;
      sc[static_cast<size_t>(L) * L] = __float2half_rn(sv - __half2float(hi));
    } else {
      out[static_cast<size_t>(clip) * L * L + e] = v;
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
  if (!(L == 128 || L == 160) || 4 * hb >= L) return false;  // the first pass prunes r = 4 .. 11
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
    case 160:
      field_fused_kernel<160><<<g, kFusedThreads, sm, st>>>(kband, Mband, K, hb, groups, keep, flare, mean, out, sp,
                                                             part, tw);
      break;
    default:
      return cudaErrorInvalidValue;
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
