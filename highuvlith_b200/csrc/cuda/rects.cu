// Exact band spectrum of rectangle clips (HUV_INPUT_RECTS).
//
// Mask::spectrum's closed form (crates/highuvlith-core/src/mask.rs:616-657,
// 1439-1503): a separable term with intervals [a, b] in x and [c, d] in y has
// the FFT-layout coefficient
//     S(ky, kx) = N^2 phi(ky) phi(kx) (g_ky(d) - g_ky(c)) (g_kx(b) - g_kx(a)),
//     g_m(x) = e^{-2 pi i m x / L} / (-2 pi i m)  (m != 0),  g_0(x) = x / L,
//     phi(m) = e^{-i pi m (N - 1) / N}   (pixel-centre sampling, mask.rs:28-36).
// Overlapping rectangles are resolved as the reference's compress does
// (mask.rs:1365-1437): on the host, the clip's distinct y edges cut it into
// rows; each row's covered x cells merge into runs; rows with equal runs
// merge.  The union is then sum_rows Y_j(ky) X_j(kx), X_j = sum of the row's
// run terms -- a complex GEMM over rows, done on the GPU in FP64:
//   rect_row_coef: one warp per row: X_j(kx) for every band order kx (each
//     lane walks the orders lane, lane + 32, ... by a phasor recurrence from
//     two sincos per run) and Y_j(ky);
//   rect_band_gemm: per clip and block of band rows ky, M(ky, kx) =
//     (feature - background) sum_j Y_j(ky) X_j(kx) (+ background N^2 at DC),
//     rows staged through shared memory; the block's share of the flare mean
//     sum W |M|^2 goes to a fixed slot (summed in order by mean_reduce).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../engine.hpp"

namespace huv_dev {

struct RectRowDev {
  double y0, y1;
  int32_t first, count;  // runs[first .. first + count)
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Sum over intervals [a_r, b_r] of (g_m(b) - g_m(a)) for m = m0 + 32 i,
// i < cnt, accumulated into acc[i] (L-normalised).
__device__ void run_terms(const double2* __restrict__ runs, int first, int count, double L, int m0, int cnt,
                          double2* acc) {
  const double two_pi = 6.283185307179586476925;
  for (int r = 0; r < count; ++r) {
    const double2 ab = runs[first + r];
    // e^{-2 pi i m x / L} at m = m0 and the step e^{-2 pi i 32 x / L}, x = a, b
    double sa0, ca0, sb0, cb0, sas, cas, sbs, cbs;
    sincospi(-2.0 * m0 * ab.x / L, &sa0, &ca0);
    sincospi(-2.0 * m0 * ab.y / L, &sb0, &cb0);
    sincospi(-64.0 * ab.x / L, &sas, &cas);
    sincospi(-64.0 * ab.y / L, &sbs, &cbs);
    double2 ea = make_double2(ca0, sa0), eb = make_double2(cb0, sb0);
    const double2 sa = make_double2(cas, sas), sb = make_double2(cbs, sbs);
    for (int i = 0; i < cnt; ++i) {
      const int m = m0 + 32 * i;
      if (m == 0) {
        acc[i].x += (ab.y - ab.x) / L;
      } else {
        // (eb - ea) / (-2 pi i m) = i (eb - ea) / (2 pi m)
        const double f = 1.0 / (two_pi * m);
        acc[i].x += -(eb.y - ea.y) * f;
        acc[i].y += (eb.x - ea.x) * f;
      }
      ea = zmul(ea, sa);
      eb = zmul(eb, sb);
    }
  }
}

// X[j][m + h] and Y[j][m + h] for every row j (one warp per row).
__global__ void rect_row_coef(const RectRowDev* __restrict__ rows, const double2* __restrict__ runs, int n_rows,
                              int h, double L, double2* __restrict__ X, double2* __restrict__ Y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n_rows) return;
  const int B = 2 * h + 1;
  const int m0 = -h + lane;
  const int cnt = m0 <= h ? (h - m0) / 32 + 1 : 0;
  double2 ax[8], ay[8];  // B <= 255 -> at most 8 orders per lane
#pragma unroll
  for (int i = 0; i < 8; ++i) ax[i] = ay[i] = make_double2(0.0, 0.0);
  const RectRowDev rw = rows[warp];
  if (cnt > 0) {
    run_terms(runs, rw.first, rw.count, L, m0, cnt, ax);
    const double2 yr = make_double2(rw.y0, rw.y1);
    run_terms(&yr, 0, 1, L, m0, cnt, ay);
  }
  for (int i = 0; i < cnt; ++i) {
    const int k = m0 + 32 * i + h;
    X[static_cast<size_t>(warp) * B + k] = ax[i];
    Y[static_cast<size_t>(warp) * B + k] = ay[i];
  }
}

// M(ky, kx) for clip c0 + blockIdx.y, band rows ky in [blockIdx.x * TY, +TY).
// Thread t owns (ky, kx) pairs t, t + 256, ... of the tile; rows staged 16 at
// a time.  Dynamic shared memory: 16 * (TY + B) double2.
constexpr int kRectTY = 16;
__global__ void __launch_bounds__(256) rect_band_gemm(const int32_t* __restrict__ clip_rows,
                                                       const double2* __restrict__ X, const double2* __restrict__ Y,
                                                       int c0, int h, int n, double2 dv, double2 bgn2,
                                                       const float* __restrict__ W, float2* __restrict__ Mband,
                                                       float* __restrict__ parts) {
  extern __shared__ double2 rs[];
  constexpr int TY = kRectTY, MAXE = (TY * 255 + 255) / 256;
  const int B = 2 * h + 1;
  const int clip = blockIdx.y, cg = c0 + clip;
  const int ky0 = blockIdx.x * TY;
  const int ty = min(TY, B - ky0);
  double2* sy = rs;               // [16][TY]
  double2* sx = rs + 16 * TY;     // [16][B]
  const int j0 = clip_rows[cg], j1 = clip_rows[cg + 1];
  const int nout = ty * B;
  double2 acc[MAXE];
#pragma unroll
  for (int e = 0; e < MAXE; ++e) acc[e] = make_double2(0.0, 0.0);
  for (int jb = j0; jb < j1; jb += 16) {
    const int nj = min(16, j1 - jb);
    __syncthreads();
    for (int t = threadIdx.x; t < nj * B; t += blockDim.x) {
      const int jj = t / B, k = t - jj * B;
      sx[jj * B + k] = X[static_cast<size_t>(jb + jj) * B + k];
    }
    for (int t = threadIdx.x; t < nj * ty; t += blockDim.x) {
      const int jj = t / ty, k = t - jj * ty;
      sy[jj * TY + k] = Y[static_cast<size_t>(jb + jj) * B + ky0 + k];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < MAXE; ++e) {
      const int o = threadIdx.x + 256 * e;
      if (o < nout) {
        const int r = o / B, kx = o - r * B;
        double2 a = acc[e];
        for (int jj = 0; jj < nj; ++jj) {
          const double2 yv = sy[jj * TY + r], xv = sx[jj * B + kx];
          a.x = fma(yv.x, xv.x, fma(-yv.y, xv.y, a.x));
          a.y = fma(yv.x, xv.y, fma(yv.y, xv.x, a.y));
        }
        acc[e] = a;
      }
    }
  }
  // scale, DC, store, flare-mean partial
  __shared__ float red[8];
  float wsum = 0.f;
  const double n2 = static_cast<double>(n) * n;
#pragma unroll
  for (int e = 0; e < MAXE; ++e) {
    const int o = threadIdx.x + 256 * e;
    if (o < nout) {
      const int r = o / B, kx = o - r * B;
      const int my = ky0 + r;
      const int qy = my - h, qx = kx - h;
      // N^2 phi(qy) phi(qx), phi(m) = e^{-i pi m (N - 1) / N}
      double s, c;
      sincospi(-static_cast<double>(qy + qx) * (n - 1) / n, &s, &c);
      const double2 ph = make_double2(c * n2, s * n2);
      double2 v = zmul(zmul(acc[e], ph), dv);
      if (qy == 0 && qx == 0) {
        v.x += bgn2.x;
        v.y += bgn2.y;
      }
      const float2 f = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
      Mband[(static_cast<size_t>(clip) * B + my) * B + kx] = f;
      if (W) wsum += W[my * B + kx] * (f.x * f.x + f.y * f.y);
    }
  }
  if (parts) {
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = wsum;
    __syncthreads();
    if (threadIdx.x == 0) {
      float t = 0.f;
      for (int w = 0; w < 8; ++w) t += red[w];
      parts[static_cast<size_t>(clip) * gridDim.x + blockIdx.x] = t;
    }
  }
}

// mean[c] = sum_i parts[c][i] in order (deterministic).
__global__ void rect_mean_reduce(const float* __restrict__ parts, int nparts, int clips, float* __restrict__ mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= clips) return;
  float s = 0.f;
  for (int i = 0; i < nparts; ++i) s += parts[static_cast<size_t>(c) * nparts + i];
  mean[c] = s;
}

}  // namespace huv_dev

namespace huv {

namespace {

// Rows of disjoint x runs for every clip (host, FP64).
void decompose(const huv_rect_clips& in, int n_clips, double L, std::vector<int32_t>& clip_rows,
               std::vector<huv_dev::RectRowDev>& rows, std::vector<double2>& runs) {
  const double half = L / 2.0;
  clip_rows.assign(1, 0);
  for (int c = 0; c < n_clips; ++c) {
    const int b = in.offsets[c], e = in.offsets[c + 1];
    struct R {
      double x0, x1, y0, y1;
    };
    std::vector<R> rs;
    std::vector<double> xe, ye;
    for (int i = b; i < e; ++i) {
      const huv_rect& q = in.rects[i];
      const double x0 = std::max(q.x - q.w / 2.0, -half), x1 = std::min(q.x + q.w / 2.0, half);
      const double y0 = std::max(q.y - q.h / 2.0, -half), y1 = std::min(q.y + q.h / 2.0, half);
      if (!(x1 > x0) || !(y1 > y0)) continue;
      rs.push_back(R{x0, x1, y0, y1});
      xe.push_back(x0);
      xe.push_back(x1);
      ye.push_back(y0);
      ye.push_back(y1);
    }
    std::sort(xe.begin(), xe.end());
    xe.erase(std::unique(xe.begin(), xe.end()), xe.end());
    std::sort(ye.begin(), ye.end());
    ye.erase(std::unique(ye.begin(), ye.end()), ye.end());
    const int E = static_cast<int>(xe.size());
    std::vector<int> cover(std::max(E - 1, 0));
    std::vector<double2> prev;
    for (size_t f = 0; f + 1 < ye.size(); ++f) {
      const double ya = ye[f], yb = ye[f + 1];
      std::fill(cover.begin(), cover.end(), 0);
      for (const R& r : rs)
        if (r.y0 <= ya && r.y1 >= yb) {
          const int e0 = static_cast<int>(std::lower_bound(xe.begin(), xe.end(), r.x0) - xe.begin());
          const int e1 = static_cast<int>(std::lower_bound(xe.begin(), xe.end(), r.x1) - xe.begin());
          for (int q = e0; q < e1; ++q) cover[q] = 1;
        }
      std::vector<double2> row;
      for (int q = 0; q + 1 < E;) {
        if (!cover[q]) {
          ++q;
          continue;
        }
        int q1 = q;
        while (q1 + 1 < E && cover[q1]) ++q1;
        row.push_back(make_double2(xe[q], xe[q1]));
        q = q1;
      }
      const bool same = !rows.empty() && static_cast<int>(rows.size()) > clip_rows.back() && row.size() == prev.size() &&
                        rows.back().y1 == ya &&
                        std::equal(row.begin(), row.end(), prev.begin(),
                                   [](const double2& u, const double2& v) { return u.x == v.x && u.y == v.y; });
      if (row.empty()) {
        prev.clear();
        continue;
      }
      if (same) {
        rows.back().y1 = yb;
      } else {
        huv_dev::RectRowDev rr{ya, yb, static_cast<int32_t>(runs.size()), static_cast<int32_t>(row.size())};
        rows.push_back(rr);
        runs.insert(runs.end(), row.begin(), row.end());
      }
      prev = row;
    }
    clip_rows.push_back(static_cast<int32_t>(rows.size()));
  }
}

}  // namespace

void Engine::upload_rects(const huv_batch& b) {
  const auto* in = static_cast<const huv_rect_clips*>(b.input);
  if (!in || !in->offsets || (in->offsets[b.n_clips] > in->offsets[0] && !in->rects))
    throw Error(HUV_ERR_INVALID_PARAMETER, "rect clips: null pointer");
  if (in->offsets[0] < 0) throw Error(HUV_ERR_INVALID_PARAMETER, "rect clips: offsets must be >= 0");
  for (int c = 0; c < b.n_clips; ++c)
    if (in->offsets[c + 1] < in->offsets[c]) throw Error(HUV_ERR_INVALID_PARAMETER, "rect clips: offsets decrease");
  for (int i = in->offsets[0]; i < in->offsets[b.n_clips]; ++i) {
    const huv_rect& q = in->rects[i];
    if (!(std::isfinite(q.x) && std::isfinite(q.y) && std::isfinite(q.w) && std::isfinite(q.h)) || q.w < 0 ||
        q.h < 0)
      throw Error(HUV_ERR_INVALID_PARAMETER, "rect clips: coordinates must be finite, sizes >= 0");
  }
  if (!(std::isfinite(in->feature_re) && std::isfinite(in->feature_im) && std::isfinite(in->background_re) &&
        std::isfinite(in->background_im)))
    throw Error(HUV_ERR_INVALID_PARAMETER, "rect clips: amplitudes must be finite");
  std::vector<int32_t> clip_rows;
  std::vector<huv_dev::RectRowDev> rows;
  std::vector<double2> runs;
  decompose(*in, b.n_clips, n * pixel_nm, clip_rows, rows, runs);
  rect.n_rows = static_cast<int>(rows.size());
  auto grow = [](void*& p, size_t& cap, size_t bytes) {
    if (bytes <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    check_cuda(cudaMalloc(&p, bytes), "cudaMalloc(rect table)");
    cap = bytes;
  };
  grow(rect.clip_rows, rect.clip_rows_cap, sizeof(int32_t) * clip_rows.size());
  grow(rect.rows, rect.rows_cap, sizeof(huv_dev::RectRowDev) * std::max<size_t>(rows.size(), 1));
  grow(rect.runs, rect.runs_cap, sizeof(double2) * std::max<size_t>(runs.size(), 1));
  check_cuda(cudaMemcpy(rect.clip_rows, clip_rows.data(), sizeof(int32_t) * clip_rows.size(), cudaMemcpyHostToDevice),
             "upload rect rows");
  if (!rows.empty()) {
    check_cuda(cudaMemcpy(rect.rows, rows.data(), sizeof(huv_dev::RectRowDev) * rows.size(), cudaMemcpyHostToDevice),
               "upload rect rows");
    check_cuda(cudaMemcpy(rect.runs, runs.data(), sizeof(double2) * runs.size(), cudaMemcpyHostToDevice),
               "upload rect runs");
  }
  rect.dv = make_double2(in->feature_re - in->background_re, in->feature_im - in->background_im);
  rect.bg = make_double2(in->background_re, in->background_im);
}

void Engine::rect_band(int c0, int nc, int hb, const float* W, float2* Mband, float* mean, cudaStream_t st) {
  const int B = 2 * hb + 1;
  if (B > 255) throw Error(HUV_ERR_UNSUPPORTED, "rect clips: band wider than 255 orders");
  const double L = n * pixel_nm;
  // Coefficients of every row of the batch (rows of later chunks are cheap
  // to recompute; the table is per batch).
  const size_t need = sizeof(double2) * 2 * static_cast<size_t>(std::max(rect.n_rows, 1)) * B;
  if (need > rect.coef_cap) {
    if (rect.coef) cudaFree(rect.coef);
    rect.coef = nullptr;
    rect.coef_cap = 0;
    check_cuda(cudaMalloc(&rect.coef, need), "cudaMalloc(rect coefficients)");
    rect.coef_cap = need;
  }
  double2* X = static_cast<double2*>(rect.coef);
  double2* Y = X + static_cast<size_t>(std::max(rect.n_rows, 1)) * B;
  if (c0 == 0 && rect.n_rows > 0) {
    const int threads = 256, warps = threads / 32;
    huv_dev::rect_row_coef<<<(rect.n_rows + warps - 1) / warps, threads, 0, st>>>(
        static_cast<const huv_dev::RectRowDev*>(rect.rows), static_cast<const double2*>(rect.runs), rect.n_rows, hb,
        L, X, Y);
    check_cuda(cudaGetLastError(), "rect_row_coef");
  }
  const int tiles = (B + huv_dev::kRectTY - 1) / huv_dev::kRectTY;
  float* parts = (W && mean) ? mean + nc : nullptr;
  const double n2 = static_cast<double>(n) * n;
  const size_t sm = sizeof(double2) * 16 * (huv_dev::kRectTY + B);
  huv_dev::rect_band_gemm<<<dim3(tiles, nc), 256, sm, st>>>(
      static_cast<const int32_t*>(rect.clip_rows), X, Y, c0, hb, n, rect.dv,
      make_double2(rect.bg.x * n2, rect.bg.y * n2), W, Mband, parts);
  check_cuda(cudaGetLastError(), "rect_band_gemm");
  if (parts) {
    huv_dev::rect_mean_reduce<<<(nc + 127) / 128, 128, 0, st>>>(parts, tiles, nc, mean);
    check_cuda(cudaGetLastError(), "mean_reduce(rects)");
  }
}

}  // namespace huv
