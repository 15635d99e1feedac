// Register-radix Stockham FFT over S interleaved sequences (FP32 complex).
//
// Each pass of radix R (16, 12, 10, 8, 4) loads R points of one butterfly
// into registers, applies the Stockham twiddles w^{r k}, does the R-point DFT
// in registers (16 = 4 x 4, 8 = 4 x 2, 12 = 3 x 4, 10 = 5 x 2 with their
// internal twiddles as constants) and stores R points; a length L of
// 128, 160, 192, 256 takes 2 passes, 512 and 1024 take 3, instead of
// log4(L) shared-memory round trips.  Lengths 160 = 16 x 10 and
// 192 = 16 x 12 serve evaluation grids just above 4h that a power of two
// would overshoot.  Data sit in shared memory sequence-minor:
// element i of sequence s at ((i + pad(i)) * S + s), pad(i) = i / 16 when
// S < 16, so that the lanes of a half-warp (consecutive s, then consecutive
// butterflies) touch distinct banks in every pass, including the strided
// writes of the first one.
//
// The phase functions are __host__ __device__ so that a host harness can run
// them thread by thread; a kernel calls them with a barrier between phases.
#pragma once
#include <cuda_runtime.h>

namespace huv_dev {

// W16^e = exp(DIR * 2 pi i e / 16), e in [0, 16): cos / sin of e pi / 8.
template <int DIR>
__host__ __device__ __forceinline__ float2 w16(int e) {
  constexpr float c[16] = {1.0f,
                           0.92387953251128674f,
                           0.70710678118654752f,
                           0.38268343236508977f,
                           0.0f,
                           -0.38268343236508977f,
                           -0.70710678118654752f,
                           -0.92387953251128674f,
                           -1.0f,
                           -0.92387953251128674f,
                           -0.70710678118654752f,
                           -0.38268343236508977f,
                           0.0f,
                           0.38268343236508977f,
                           0.70710678118654752f,
                           0.92387953251128674f};
  const float s = c[(e + 12) & 15];  // sin(x) = cos(x - pi/2)
  return make_float2(c[e & 15], DIR > 0 ? s : -s);
}

__host__ __device__ __forceinline__ float2 fr_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 fr_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 fr_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by exp(DIR * i pi / 2): +i (DIR > 0) or -i
template <int DIR>
__host__ __device__ __forceinline__ float2 fr_rot90(float2 a) {
  return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// 4-point DFT of (a0, a1, a2, a3) in place.
template <int DIR>
__host__ __device__ __forceinline__ void fr_dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  const float2 s02 = fr_add(a0, a2), d02 = fr_sub(a0, a2);
  const float2 s13 = fr_add(a1, a3), d13 = fr_rot90<DIR>(fr_sub(a1, a3));
  a0 = fr_add(s02, s13);
  a2 = fr_sub(s02, s13);
  a1 = fr_add(d02, d13);
  a3 = fr_sub(d02, d13);
}

// exp(DIR * 2 pi i e / N) for N = 10, 12 (e in [0, N)), from the exact
// values of cos and sin at multiples of pi / 5 and pi / 6.
template <int N, int DIR>
__host__ __device__ __forceinline__ float2 fr_w(int e) {
  float c, s;
  if constexpr (N == 10) {
    // cos / sin of e pi / 5, e = 0 .. 9
    constexpr float cs[10] = {1.0f, 0.80901699437494742f, 0.30901699437494742f, -0.30901699437494742f,
                              -0.80901699437494742f, -1.0f, -0.80901699437494742f, -0.30901699437494742f,
                              0.30901699437494742f, 0.80901699437494742f};
    constexpr float sn[10] = {0.0f, 0.58778525229247313f, 0.95105651629515357f, 0.95105651629515357f,
                              0.58778525229247313f, 0.0f, -0.58778525229247313f, -0.95105651629515357f,
                              -0.95105651629515357f, -0.58778525229247313f};
    c = cs[e % 10];
    s = sn[e % 10];
  } else {
    // cos / sin of e pi / 6, e = 0 .. 11
    constexpr float cs[12] = {1.0f, 0.86602540378443865f, 0.5f, 0.0f, -0.5f, -0.86602540378443865f,
                              -1.0f, -0.86602540378443865f, -0.5f, 0.0f, 0.5f, 0.86602540378443865f};
    constexpr float sn[12] = {0.0f, 0.5f, 0.86602540378443865f, 1.0f, 0.86602540378443865f, 0.5f,
                              0.0f, -0.5f, -0.86602540378443865f, -1.0f, -0.86602540378443865f, -0.5f};
    c = cs[e % 12];
    s = sn[e % 12];
  }
  return make_float2(c, DIR > 0 ? s : -s);
}

// multiply by DIR i: (x + i y) -> DIR (-y + i x)
template <int DIR>
__host__ __device__ __forceinline__ float2 fr_idir(float2 a) {
  return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// 3-point DFT in place: X1,2 = v0 - (v1 + v2) / 2 +- DIR i sqrt(3)/2 (v1 - v2).
template <int DIR>
__host__ __device__ __forceinline__ void fr_dft3(float2 (&v)[3]) {
  constexpr float h = 0.86602540378443865f;
  const float2 t = fr_add(v[1], v[2]);
  const float2 d = fr_sub(v[1], v[2]);
  const float2 a = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
  const float2 b = fr_idir<DIR>(make_float2(h * d.x, h * d.y));
  v[0] = fr_add(v[0], t);
  v[1] = fr_add(a, b);
  v[2] = fr_sub(a, b);
}

// 5-point DFT in place (c1, s1 = cos, sin 2 pi / 5; c2, s2 = cos, sin 4 pi / 5):
// X1,4 = v0 + c1 (v1 + v4) + c2 (v2 + v3) +- DIR i (s1 (v1 - v4) + s2 (v2 - v3)),
// X2,3 = v0 + c2 (v1 + v4) + c1 (v2 + v3) +- DIR i (s2 (v1 - v4) - s1 (v2 - v3)).
template <int DIR>
__host__ __device__ __forceinline__ void fr_dft5(float2 (&v)[5]) {
  constexpr float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
  constexpr float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;
  const float2 t1 = fr_add(v[1], v[4]), t2 = fr_add(v[2], v[3]);
  const float2 d1 = fr_sub(v[1], v[4]), d2 = fr_sub(v[2], v[3]);
  const float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  const float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  const float2 b1 = fr_idir<DIR>(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
  const float2 b2 = fr_idir<DIR>(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
  v[0] = fr_add(v[0], fr_add(t1, t2));
  v[1] = fr_add(a1, b1);
  v[4] = fr_sub(a1, b1);
  v[2] = fr_add(a2, b2);
  v[3] = fr_sub(a2, b2);
}

// R-point DFT of v in place, natural order in and out.
template <int R, int DIR>
__host__ __device__ __forceinline__ void fr_dft(float2 (&v)[R]) {
  if constexpr (R == 2) {
    const float2 a = v[0];
    v[0] = fr_add(a, v[1]);
    v[1] = fr_sub(a, v[1]);
  } else if constexpr (R == 4) {
    fr_dft4<DIR>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // n = q + 2 m, k = p + 4 q': X = sum_q W2^{q q'} W8^{q p} [sum_m v W4^{m p}]
    float2 u[2][4];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      u[q][0] = v[q];
      u[q][1] = v[q + 2];
      u[q][2] = v[q + 4];
      u[q][3] = v[q + 6];
      fr_dft4<DIR>(u[q][0], u[q][1], u[q][2], u[q][3]);
    }
#pragma unroll
    for (int p = 1; p < 4; ++p) u[1][p] = fr_mul(u[1][p], w16<DIR>(2 * p));
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      v[p] = fr_add(u[0][p], u[1][p]);
      v[p + 4] = fr_sub(u[0][p], u[1][p]);
    }
  } else if constexpr (R == 10) {
    // n = q + 2 m, k = p + 5 q': X = sum_q W2^{q q'} W10^{q p} [sum_m v W5^{m p}]
    float2 u[2][5];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
#pragma unroll
      for (int m = 0; m < 5; ++m) u[q][m] = v[q + 2 * m];
      fr_dft5<DIR>(u[q]);
    }
#pragma unroll
    for (int p = 1; p < 5; ++p) u[1][p] = fr_mul(u[1][p], fr_w<10, DIR>(p));
#pragma unroll
    for (int p = 0; p < 5; ++p) {
      v[p] = fr_add(u[0][p], u[1][p]);
      v[p + 5] = fr_sub(u[0][p], u[1][p]);
    }
  } else if constexpr (R == 12) {
    // n = q + 4 m, k = p + 3 q': X = sum_q W4^{q q'} W12^{q p} [sum_m v W3^{m p}]
    float2 u[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
      for (int m = 0; m < 3; ++m) u[q][m] = v[q + 4 * m];
      fr_dft3<DIR>(u[q]);
    }
#pragma unroll
    for (int q = 1; q < 4; ++q)
#pragma unroll
      for (int p = 1; p < 3; ++p) u[q][p] = fr_mul(u[q][p], fr_w<12, DIR>(q * p));
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      fr_dft4<DIR>(u[0][p], u[1][p], u[2][p], u[3][p]);
      v[p] = u[0][p];
      v[p + 3] = u[1][p];
      v[p + 6] = u[2][p];
      v[p + 9] = u[3][p];
    }
  } else if constexpr (R == 16) {
    // n = q + 4 m, k = p + 4 q': X = sum_q W4^{q q'} W16^{q p} [sum_m v W4^{m p}]
    float2 u[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      u[q][0] = v[q];
      u[q][1] = v[q + 4];
      u[q][2] = v[q + 8];
      u[q][3] = v[q + 12];
      fr_dft4<DIR>(u[q][0], u[q][1], u[q][2], u[q][3]);
    }
#pragma unroll
    for (int q = 1; q < 4; ++q)
#pragma unroll
      for (int p = 1; p < 4; ++p) u[q][p] = fr_mul(u[q][p], w16<DIR>(q * p));
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      fr_dft4<DIR>(u[0][p], u[1][p], u[2][p], u[3][p]);
      v[p] = u[0][p];
      v[p + 4] = u[1][p];
      v[p + 8] = u[2][p];
      v[p + 12] = u[3][p];
    }
  }
}

// 16-point DFT of v in place when v[4] .. v[11] are zero (not read): the
// inner 4-point DFTs of the 4 x 4 split (n = q + 4 m) have inputs m = 0 and
// m = 3 only, X_q = (a0 + a3, a0 - i a3, a0 - a3, a0 + i a3) for the
// direction's i, then the twiddles and outer DFTs of fr_dft<16>.  The first
// pass over a zero-padded band of half-width h < L / 4 has exactly this
// shape: its inputs j + r L / 16 with 4 <= r <= 11 lie outside the band.
template <int DIR>
__host__ __device__ __forceinline__ void fr_dft16_band(float2 (&v)[16]) {
  float2 u[4][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 a0 = v[q], a3 = v[q + 12];
    const float2 t = fr_rot90<DIR>(a3);
    u[q][0] = fr_add(a0, a3);
    u[q][1] = fr_sub(a0, t);
    u[q][2] = fr_sub(a0, a3);
    u[q][3] = fr_add(a0, t);
  }
#pragma unroll
  for (int q = 1; q < 4; ++q)
#pragma unroll
    for (int p = 1; p < 4; ++p) u[q][p] = fr_mul(u[q][p], w16<DIR>(q * p));
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    fr_dft4<DIR>(u[0][p], u[1][p], u[2][p], u[3][p]);
    v[p] = u[0][p];
    v[p + 4] = u[1][p];
    v[p + 8] = u[2][p];
    v[p + 12] = u[3][p];
  }
}

// Radix plan by length: 128 = 16 x 8, 160 = 16 x 10, 192 = 16 x 12,
// 256 = 16 x 16, 384 = 16 x 12 x 2, 512 = 16 x 8 x 4, 1024 = 16 x 16 x 4,
// 2048 = 16 x 16 x 8.
__host__ __device__ constexpr int fr_passes(int L) { return L <= 256 ? 2 : 3; }
__host__ __device__ constexpr int fr_radix(int L, int pass) {
  return pass == 0 ? 16
         : L == 128 ? 8
         : L == 160 ? 10
         : L == 192 ? 12
         : L == 256 ? 16
         : L == 384 ? (pass == 1 ? 12 : 2)
         : L == 512 ? (pass == 1 ? 8 : 4)
         : L == 2048 ? (pass == 1 ? 16 : 8)
                     : (pass == 1 ? 16 : 4);
}
// Stockham sub-transform size before pass `pass`.
__host__ __device__ constexpr int fr_ns(int L, int pass) {
  return pass == 0 ? 1 : fr_ns(L, pass - 1) * fr_radix(L, pass - 1);
}

// Shared-memory index of element i of sequence s.
template <int S>
__host__ __device__ __forceinline__ int fr_idx(int i, int s) {
  return (S < 16 ? i + (i >> 4) : i) * S + s;
}
// Buffer length (float2) for S sequences of length L.
__host__ __device__ constexpr int fr_buf(int L, int S) { return (S < 16 ? L + L / 16 : L) * S; }

// Threads of one block (256 for every plan), butterflies of pass `pass`
// over S sequences, and butterflies per thread (rounded up; the last round
// is guarded where the count is not a multiple of 256).
__host__ __device__ constexpr int fr_threads(int L, int S) { return (void)L, (void)S, 256; }
__host__ __device__ constexpr int fr_nb(int L, int S, int pass) { return S * L / fr_radix(L, pass); }
__host__ __device__ constexpr int fr_per(int L, int S, int pass) {
  return (fr_nb(L, S, pass) + fr_threads(L, S) - 1) / fr_threads(L, S);
}

// Asynchronous 8-byte global -> shared copies (cp.async, L1-allocating) for
// prefetching the next kernel's band columns while the current one is
// transformed.
__device__ __forceinline__ void fr_cp_async8(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(smem_dst))),
               "l"(gmem_src)
               : "memory");
}
// 16-byte variant (L2 only): both addresses 16-byte aligned.
__device__ __forceinline__ void fr_cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(smem_dst))),
               "l"(gmem_src)
               : "memory");
}
__device__ __forceinline__ void fr_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void fr_cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Sequences per block of the register-radix kernels for length L (256
// threads each), 0 where no instance exists; shared-memory bytes of the
// ping-pong buffers of one block and the kernels' shared-memory ceiling.
__host__ __device__ constexpr int xt_S(int L) {
  return L == 128 ? 32
         : (L == 160 || L == 192 || L == 256) ? 16
         : (L == 384 || L == 512) ? 8
         : L == 1024 ? 4
         : L == 2048 ? 2
                     : 0;
}
__host__ __device__ constexpr size_t xt_buf_bytes(int L) {
  // one buffer: the middle passes run in place (fr_mid_pass_inplace)
  return xt_S(L) ? static_cast<size_t>(fr_buf(L, xt_S(L))) * sizeof(float2) : 0;
}
constexpr int kXtSmemMax = 110 * 1024;

// First pass (radix 16, no twiddles) for thread t, reading a zero-padded
// band: position i of sequence s holds P[s][mx] for the order mx - hb = i
// (i <= hb) or i - L (i >= L - hb), and zero elsewhere.  Requires 2 hb < L.
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_first_pass_band(int t, const float2* P, int B, int hb, float2* dst) {
  if (t >= fr_nb(L, S, 0)) return;
  const int s = t % S, j = t / S;
  float2 v[16];
  if (4 * hb < L) {
    // inputs r = 4 .. 11 lie outside the band: 8 loads and the pruned DFT
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      if (r >= 4 && r < 12) continue;
      const int i = j + r * (L / 16);
      const int mx = r < 4 ? (i <= hb ? i + hb : -1) : (i >= L - hb ? i - L + hb : -1);
      v[r] = mx >= 0 ? P[s * B + mx] : make_float2(0.f, 0.f);
    }
    fr_dft16_band<DIR>(v);
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int i = j + r * (L / 16);
      const int mx = i <= hb ? i + hb : (i >= L - hb ? i - L + hb : -1);
      v[r] = mx >= 0 ? P[s * B + mx] : make_float2(0.f, 0.f);
    }
    fr_dft<16, DIR>(v);
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[fr_idx<S>(j * 16 + r, s)] = v[r];
}

// The pruned band first pass (4 hb < L) with its input offsets computed
// once: off[q] is the index into P (sequence s's band row, s B + mx) of
// input r = q (q < 4) or r = q + 8 (q >= 4), -1 where it lies outside the
// band.  The offsets depend only on the thread, so a kernel that runs the
// pass for many band blocks (one per SOCS kernel) computes them once.
template <int L, int S>
__host__ __device__ __forceinline__ void fr_band_offsets(int t, int B, int hb, int (&off)[8]) {
  const int s = t % S, j = t / S;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int r = q < 4 ? q : q + 8;
    const int i = j + r * (L / 16);
    const int mx = r < 4 ? (i <= hb ? i + hb : -1) : (i >= L - hb ? i - L + hb : -1);
    off[q] = mx >= 0 ? s * B + mx : -1;
  }
}
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_first_pass_band_off(int t, const float2* P, const int (&off)[8],
                                                                float2* dst) {
  if (t >= fr_nb(L, S, 0)) return;
  const int s = t % S, j = t / S;
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q < 4 ? q : q + 8] = off[q] >= 0 ? P[off[q]] : make_float2(0.f, 0.f);
  fr_dft16_band<DIR>(v);
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[fr_idx<S>(j * 16 + r, s)] = v[r];
}

// First pass (radix 16, no twiddles) for thread t given its 16 inputs
// v[r] = element j + r L / 16 of sequence s (s = t % S, j = t / S).
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_first_pass_vals(int t, float2 (&v)[16], float2* dst) {
  if (t >= fr_nb(L, S, 0)) return;
  const int s = t % S, j = t / S;
  fr_dft<16, DIR>(v);
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[fr_idx<S>(j * 16 + r, s)] = v[r];
}

// Middle pass `pass` (not the first, not the last) for thread t: src -> dst.
template <int L, int S, int DIR, int PASS>
__host__ __device__ __forceinline__ void fr_mid_pass(int t, const float2* src, float2* dst, const float2* tw) {
  constexpr int R = fr_radix(L, PASS), Ns = fr_ns(L, PASS), T = fr_threads(L, S);
  constexpr int stride = L / (Ns * R);
#pragma unroll
  for (int b = 0; b < fr_per(L, S, PASS); ++b) {
    const int u = t + b * T;
    if (u >= fr_nb(L, S, PASS)) break;
    const int s = u % S, j = u / S;
    const int k = j % Ns;  // Ns need not be a power of two (384 = 16 x 12 x 2)
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[fr_idx<S>(j + r * (L / R), s)];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 w = tw[r * k * stride];
      if (DIR > 0) w.y = -w.y;
      v[r] = fr_mul(v[r], w);
    }
    fr_dft<R, DIR>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[fr_idx<S>(base + r * Ns, s)] = v[r];
  }
}

// Middle pass `pass` in place: every thread loads the inputs of all its
// butterflies, the block synchronises, then every thread transforms and
// stores into the same buffer (one FFT buffer per block instead of two, so
// more blocks fit an SM).  Called by all threads of the block.
template <int L, int S, int DIR, int PASS>
__device__ __forceinline__ void fr_mid_pass_inplace(int t, float2* buf, const float2* tw) {
  constexpr int R = fr_radix(L, PASS), Ns = fr_ns(L, PASS), T = fr_threads(L, S), PER = fr_per(L, S, PASS);
  constexpr int stride = L / (Ns * R);
  float2 v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int u = t + b * T;
    if (u >= fr_nb(L, S, PASS)) break;
    const int s = u % S, j = u / S;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b][r] = buf[fr_idx<S>(j + r * (L / R), s)];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int u = t + b * T;
    if (u >= fr_nb(L, S, PASS)) break;
    const int s = u % S, j = u / S;
    const int k = j % Ns;  // Ns need not be a power of two (384 = 16 x 12 x 2)
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 w = tw[r * k * stride];
      if (DIR > 0) w.y = -w.y;
      v[b][r] = fr_mul(v[b][r], w);
    }
    fr_dft<R, DIR>(v[b]);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[fr_idx<S>(base + r * Ns, s)] = v[b][r];
  }
}

// Last pass for butterfly u: loads, twiddles and transforms; returns the
// sequence s and j; v[p] is output element x = j + p * (L / R).
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_last_pass(int u, const float2* src, const float2* tw, int& s, int& j,
                                                      float2 (&v)[fr_radix(L, fr_passes(L) - 1)]) {
  constexpr int P = fr_passes(L) - 1;
  constexpr int R = fr_radix(L, P), Ns = fr_ns(L, P);
  constexpr int stride = L / (Ns * R);  // 1
  s = u % S;
  j = u / S;
  const int k = j;  // j < L / R = Ns
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = src[fr_idx<S>(j + r * (L / R), s)];
#pragma unroll
  for (int r = 1; r < R; ++r) {
    float2 w = tw[r * k * stride];
    if (DIR > 0) w.y = -w.y;
    v[r] = fr_mul(v[r], w);
  }
  fr_dft<R, DIR>(v);
}

// The last pass's twiddles of thread t (for each of its 16 / R butterflies,
// w^{r j} for r = 1 .. R - 1, direction applied): they depend only on t, so
// kernels that run the same transform shape many times load them once.
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_last_twiddles(
    int t, const float2* tw,
    float2 (&w)[fr_per(L, S, fr_passes(L) - 1)][fr_radix(L, fr_passes(L) - 1) - 1]) {
  constexpr int P = fr_passes(L) - 1;
  constexpr int R = fr_radix(L, P), T = fr_threads(L, S);
#pragma unroll
  for (int b = 0; b < fr_per(L, S, P); ++b) {
    const int j = ((t + b * T) / S) % (L / R);  // guarded butterflies: any valid index
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 x = tw[r * j];
      if (DIR > 0) x.y = -x.y;
      w[b][r - 1] = x;
    }
  }
}

// fr_last_pass with the twiddles of butterfly b preloaded (fr_last_twiddles).
template <int L, int S, int DIR>
__host__ __device__ __forceinline__ void fr_last_pass_pre(int u, const float2* src,
                                                          const float2 (&w)[fr_radix(L, fr_passes(L) - 1) - 1],
                                                          int& s, int& j,
                                                          float2 (&v)[fr_radix(L, fr_passes(L) - 1)]) {
  constexpr int R = fr_radix(L, fr_passes(L) - 1);
  s = u % S;
  j = u / S;
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = src[fr_idx<S>(j + r * (L / R), s)];
#pragma unroll
  for (int r = 1; r < R; ++r) v[r] = fr_mul(v[r], w[r - 1]);
  fr_dft<R, DIR>(v);
}

// Scale of the coarse intensity while it is carried in FP16 split planes by
// the separable band interpolation: planes hold I / s with s = 16 mean(I),
// so their scale does not depend on the normalisation, and a non-negative
// band-limited image on M^2 points (max <= M^2 mean) stays below M^2 / 16
// (2304 at M = 192), far inside FP16's range.
__device__ __forceinline__ float interp_scale(float mean) { return 16.f * fmaxf(mean, 1e-20f); }

}  // namespace huv_dev
