// Host check of the register-radix FFT plans of csrc/cuda/fft_reg.cuh (the
// pass functions are __host__ __device__): a 256-thread block is emulated
// thread by thread, the in-place middle pass as the out-of-place pass from a
// snapshot of the buffer (the block barrier between its loads and stores
// makes the two equal), against a direct DFT in double precision.  Inputs are
// zero-padded bands of half-width hb, read through the band first pass
// (pruned when 4 hb < L).  Prints one line per case: L S DIR hb max_rel_err.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../highuvlith_b200/csrc/cuda/fft_reg.cuh"
using namespace huv_dev;

template <int L, int S, int DIR>
double run(int hb) {
  constexpr int T = 256, NP = fr_passes(L), R = fr_radix(L, NP - 1);
  std::vector<float2> tw(L), in(S * L, make_float2(0, 0)), b0(fr_buf(L, S)), snap(fr_buf(L, S)), out(S * L);
  for (int t = 0; t < L; ++t) tw[t] = make_float2((float)cos(-2 * M_PI * t / L), (float)sin(-2 * M_PI * t / L));
  const int B = 2 * hb + 1;
  std::vector<float2> P(S * B);
  srand(1234 + L + hb);
  for (int s = 0; s < S; ++s)
    for (int mx = 0; mx < B; ++mx) {
      const float2 v = make_float2(rand() / (float)RAND_MAX - 0.5f, rand() / (float)RAND_MAX - 0.5f);
      P[s * B + mx] = v;
      in[s * L + (mx - hb < 0 ? mx - hb + L : mx - hb)] = v;
    }
  for (int t = 0; t < T; ++t) fr_first_pass_band<L, S, DIR>(t, P.data(), B, hb, b0.data());
  if (NP == 3) {
    snap = b0;
    for (int t = 0; t < T; ++t) fr_mid_pass<L, S, DIR, 1>(t, snap.data(), b0.data(), tw.data());
  }
  for (int t = 0; t < T; ++t)
    for (int b = 0; b < fr_per(L, S, NP - 1); ++b) {
      if (t + b * T >= fr_nb(L, S, NP - 1)) break;
      int s, j;
      float2 v[R];
      fr_last_pass<L, S, DIR>(t + b * T, b0.data(), tw.data(), s, j, v);
      for (int p = 0; p < R; ++p) out[s * L + j + p * (L / R)] = v[p];
    }
  double worst = 0, mag = 0;
  for (int s = 0; s < S; s += (S > 4 ? S / 4 : 1))
    for (int k = 0; k < L; ++k) {
      double re = 0, im = 0;
      for (int x = 0; x < L; ++x) {
        const double a = DIR * 2 * M_PI * (double)x * k / L;
        re += in[s * L + x].x * cos(a) - in[s * L + x].y * sin(a);
        im += in[s * L + x].x * sin(a) + in[s * L + x].y * cos(a);
      }
      worst = fmax(worst, fabs(re - out[s * L + k].x) + fabs(im - out[s * L + k].y));
      mag = fmax(mag, fabs(re) + fabs(im));
    }
  return worst / mag;
}

// The form band_rows_reg uses: the first pass on full inputs, then every
// later pass as a middle pass (the last one leaves natural order in the
// buffer).
template <int L, int S, int DIR>
double run_all_mid() {
  constexpr int T = 256, NP = fr_passes(L);
  std::vector<float2> tw(L), in(S * L), b0(fr_buf(L, S)), snap(fr_buf(L, S));
  for (int t = 0; t < L; ++t) tw[t] = make_float2((float)cos(-2 * M_PI * t / L), (float)sin(-2 * M_PI * t / L));
  srand(99 + L);
  for (auto& v : in) v = make_float2(rand() / (float)RAND_MAX - 0.5f, rand() / (float)RAND_MAX - 0.5f);
  for (int t = 0; t < T; ++t) {
    if (t >= fr_nb(L, S, 0)) continue;
    const int s = t % S, j = t / S;
    float2 v[16];
    for (int r = 0; r < 16; ++r) v[r] = in[s * L + j + r * (L / 16)];
    fr_first_pass_vals<L, S, DIR>(t, v, b0.data());
  }
  snap = b0;
  for (int t = 0; t < T; ++t) fr_mid_pass<L, S, DIR, 1>(t, snap.data(), b0.data(), tw.data());
  if (NP == 3) {
    snap = b0;
    for (int t = 0; t < T; ++t) fr_mid_pass<L, S, DIR, 2>(t, snap.data(), b0.data(), tw.data());
  }
  double worst = 0, mag = 0;
  for (int s = 0; s < S; s += (S > 4 ? S / 4 : 1))
    for (int k = 0; k < L; ++k) {
      double re = 0, im = 0;
      for (int x = 0; x < L; ++x) {
        const double a = DIR * 2 * M_PI * (double)x * k / L;
        re += in[s * L + x].x * cos(a) - in[s * L + x].y * sin(a);
        im += in[s * L + x].x * sin(a) + in[s * L + x].y * cos(a);
      }
      const float2 o = b0[fr_idx<S>(k, s)];
      worst = fmax(worst, fabs(re - o.x) + fabs(im - o.y));
      mag = fmax(mag, fabs(re) + fabs(im));
    }
  return worst / mag;
}

template <int L>
void both(int hb) {
  constexpr int S = xt_S(L);
  printf("%d %d -1 %d %.3e\n", L, S, hb, run<L, S, -1>(hb));
  printf("%d %d 1 %d %.3e\n", L, S, hb, run<L, S, +1>(hb));
}

int main() {
  both<128>(31);   // pruned: 4 hb < L
  both<128>(40);   // full first pass
  both<160>(37);
  both<160>(45);
  both<192>(47);
  both<256>(63);
  both<384>(95);
  both<384>(100);
  both<512>(95);
  both<1024>(47);
  both<1024>(300);
  both<2048>(95);
  printf("rows 160 %d -1 0 %.3e\n", xt_S(160), run_all_mid<160, xt_S(160), -1>());
  printf("rows 192 %d -1 0 %.3e\n", xt_S(192), run_all_mid<192, xt_S(192), -1>());
  printf("rows 384 %d -1 0 %.3e\n", xt_S(384), run_all_mid<384, xt_S(384), -1>());
  printf("rows 1024 %d -1 0 %.3e\n", xt_S(1024), run_all_mid<1024, xt_S(1024), -1>());
  printf("rows 2048 %d -1 0 %.3e\n", xt_S(2048), run_all_mid<2048, xt_S(2048), -1>());
  return 0;
}
