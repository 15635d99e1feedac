// FP64 SOCS kernel construction on the device.
//
// Same mathematics as the host build (KernelBuilder::build,
// crates/highuvlith-core/src/aerial.rs:1041-1317): A[f, s] = sqrt(w_s)
// P((f + s) / f_c) over the candidate orders f and source points s, then the
// leading eigenpairs of TCC = A A^H.  The A fill and every product with A run
// on the GPU in FP64; only matrices of the retained rank (or the dense
// Hermitian matrix for the eigensolver) visit the host.
//
// Two solvers:
//  * dense: TCC (rows of A that some point reaches) or Gram A^H A (kept
//    columns), whichever is smaller, formed on the device; the Hermitian
//    eigensolve runs on the host; Gram vectors are mapped back (u = A v /
//    sqrt(lambda)) on the device.  Identical in exact arithmetic to the host
//    build.
//  * randomized subspace iteration with the reference's parameters (subspace
//    max_kernels + 16, 3 power iterations, linalg.rs:657-679), used when the
//    reference's rule picks it (aerial.rs:1116-1128): Q = orth(A Omega), then
//    3 x {Z = orth(A^H Q), Q = orth(A Z)}, T = (A^H Q)^H (A^H Q), eig T = W L W^H,
//    U = Q W.  Orthonormalisation is Cholesky-QR applied twice (the Gram
//    factor is l x l, on the host), with a host modified Gram-Schmidt fallback
//    for a rank-deficient block.  Omega is drawn from this file's own
//    counter-based generator (the reference's StdRng stream is not
//    reproduced; both are random starts of the same iteration).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "../engine.hpp"

namespace huv_dev {

struct DevOptics {
  int kind;
  double na, medium, obscuration, amp;
  int paraxial;
};

__device__ double kb_defocus_phase(double z, double na_rho, double medium, double lambda, int paraxial) {
  const double pi = 3.14159265358979323846;
  const double s = na_rho / medium;
  const double s2 = s * s;
  if (paraxial) return pi * z * medium * s2 / lambda;
  const double c = sqrt(fmax(1.0 - s2, 0.0));
  return 2.0 * pi * medium * z * s2 / ((1.0 + c) * lambda);
}

// The scalar pupil of Optics::pupil (host), FP64.
__device__ double2 kb_pupil(const DevOptics& o, double fx, double fy, double z, double lambda) {
  const double rho2 = fx * fx + fy * fy;
  if (rho2 > 1.0) return make_double2(0.0, 0.0);
  const double rho = sqrt(rho2);
  if (o.kind == HUV_OPTICS_EUV) {
    if (rho < o.obscuration) return make_double2(0.0, 0.0);
    const double ph = (z == 0.0) ? 0.0 : kb_defocus_phase(z, o.na * rho, 1.0, lambda, o.paraxial);
    double s, c;
    sincos(ph, &s, &c);
    return make_double2(o.amp * c, o.amp * s);
  }
  const double ph = (z == 0.0) ? 0.0 : kb_defocus_phase(z, o.na * rho, o.medium, lambda, o.paraxial);
  double s, c;
  sincos(ph, &s, &c);
  return make_double2(c, s);
}

// A (column-major rows x cols): A[r + c * rows] = sqrt(w_c) P(cand_r + point_c).
__global__ void kb_fill_a(DevOptics o, const double2* __restrict__ cand, const double3* __restrict__ pts, int rows,
                          int cols, double z, double lambda, double2* __restrict__ A) {
  const size_t total = static_cast<size_t>(rows) * cols;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t % rows), c = static_cast<int>(t / rows);
    const double3 p = pts[c];
    const double2 v = kb_pupil(o, cand[r].x + p.x, cand[r].y + p.y, z, lambda);
    const double a = sqrt(p.z);
    A[t] = make_double2(v.x * a, v.y * a);
  }
}

// C (m x n, column-major, ldc) = op(A) op(B); op(X) = X (tr = 0) or X^H
// (tr = 1); op(A) is m x k, op(B) is k x n.  32 x 32 output tiles, 256
// threads with 2 x 2 outputs each, K in steps of 16 through shared memory.
__global__ void __launch_bounds__(256) kb_zgemm(int m, int n, int k, const double2* __restrict__ A, int lda, int ta,
                                                 const double2* __restrict__ B, int ldb, int tb,
                                                 double2* __restrict__ C, int ldc) {
  __shared__ double2 sa[16][33];  // [kk][i]
  __shared__ double2 sb[16][33];  // [kk][j]
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  double2 acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b] = make_double2(0.0, 0.0);
  for (int p0 = 0; p0 < k; p0 += 16) {
    for (int e = t; e < 16 * 32; e += 256) {
      const int kk = e >> 5, ii = e & 31;
      const int i = i0 + ii, p = p0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (i < m && p < k) {
        if (ta) {
          v = A[p + static_cast<size_t>(i) * lda];
          v.y = -v.y;
        } else {
          v = A[i + static_cast<size_t>(p) * lda];
        }
      }
      sa[kk][ii] = v;
      const int j = j0 + ii;
      double2 w = make_double2(0.0, 0.0);
      if (j < n && p < k) {
        if (tb) {
          w = B[j + static_cast<size_t>(p) * ldb];
          w.y = -w.y;
        } else {
          w = B[p + static_cast<size_t>(j) * ldb];
        }
      }
      sb[kk][ii] = w;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < 16; ++kk) {
      const double2 a0 = sa[kk][tx * 2], a1 = sa[kk][tx * 2 + 1];
      const double2 b0 = sb[kk][ty * 2], b1 = sb[kk][ty * 2 + 1];
      const double2 av[2] = {a0, a1}, bv[2] = {b0, b1};
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          acc[a][b].x = fma(av[a].x, bv[b].x, fma(-av[a].y, bv[b].y, acc[a][b].x));
          acc[a][b].y = fma(av[a].x, bv[b].y, fma(av[a].y, bv[b].x, acc[a][b].y));
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int i = i0 + tx * 2 + a, j = j0 + ty * 2 + b;
      if (i < m && j < n) C[i + static_cast<size_t>(j) * ldc] = acc[a][b];
    }
}

// Column scaling: X[:, j] *= s[j].
__global__ void kb_scale_cols(double2* __restrict__ X, int rows, int cols, const double* __restrict__ s) {
  const size_t total = static_cast<size_t>(rows) * cols;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double f = s[t / rows];
    X[t].x *= f;
    X[t].y *= f;
  }
}

// Complex standard normal samples (E|z|^2 = 1) from a counter-based hash
// (SplitMix64 finaliser) and the Box-Muller transform.
__device__ __forceinline__ uint64_t kb_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__global__ void kb_gaussian(double2* __restrict__ X, size_t total, uint64_t seed) {
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint64_t a = kb_mix(seed ^ (2 * t)), b = kb_mix(seed ^ (2 * t + 1));
    const double u1 = (static_cast<double>(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
    const double u2 = static_cast<double>(b >> 11) * (1.0 / 9007199254740992.0);
    const double r = sqrt(-2.0 * log(u1)) * 0.70710678118654752;
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    X[t] = make_double2(r * c, r * s);
  }
}

}  // namespace huv_dev

namespace huv {

namespace {

using cdv = std::complex<double>;

struct Dev {
  cudaStream_t st = nullptr;
  std::vector<void*> bufs;
  explicit Dev(int device) {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate(kbuild)");
  }
  ~Dev() {
    for (void* p : bufs) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    check_cuda(cudaMallocAsync(&p, count * sizeof(T), st), "cudaMallocAsync(kbuild)");
    bufs.push_back(p);
    return static_cast<T*>(p);
  }
  template <typename T>
  void up(T* d, const T* h, size_t count) {
    check_cuda(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, st), "H2D(kbuild)");
  }
  template <typename T>
  void down(T* h, const T* d, size_t count) {
    check_cuda(cudaMemcpyAsync(h, d, count * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H(kbuild)");
    check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize(kbuild)");
  }
  // C = op(A) op(B), column-major.
  void gemm(int m, int n, int k, const double2* A, int lda, bool ta, const double2* B, int ldb, bool tb, double2* C,
            int ldc) {
    dim3 g((m + 31) / 32, (n + 31) / 32);
    huv_dev::kb_zgemm<<<g, 256, 0, st>>>(m, n, k, A, lda, ta ? 1 : 0, B, ldb, tb ? 1 : 0, C, ldc);
    check_cuda(cudaGetLastError(), "kb_zgemm");
  }
};

// Upper Cholesky factor R of a Hermitian positive definite l x l matrix G
// (column-major), G = R^H R.  Returns false if a pivot is not positive.
bool cholesky_upper(int l, const std::vector<cdv>& G, std::vector<cdv>& R) {
  R.assign(static_cast<size_t>(l) * l, cdv(0, 0));
  double gmax = 0.0;
  for (int i = 0; i < l; ++i) gmax = std::max(gmax, G[static_cast<size_t>(i) * l + i].real());
  for (int j = 0; j < l; ++j) {
    for (int i = 0; i <= j; ++i) {
      cdv s = G[static_cast<size_t>(j) * l + i];  // G(i, j)
      for (int p = 0; p < i; ++p) s -= std::conj(R[static_cast<size_t>(i) * l + p]) * R[static_cast<size_t>(j) * l + p];
      if (i == j) {
        if (!(s.real() > 1e-12 * gmax)) return false;
        R[static_cast<size_t>(j) * l + j] = std::sqrt(s.real());
      } else {
        R[static_cast<size_t>(j) * l + i] = s / R[static_cast<size_t>(i) * l + i];
      }
    }
  }
  return true;
}

// Inverse of an upper-triangular l x l matrix (column-major).
std::vector<cdv> upper_inverse(int l, const std::vector<cdv>& R) {
  std::vector<cdv> X(static_cast<size_t>(l) * l, cdv(0, 0));
  for (int j = 0; j < l; ++j) {
    X[static_cast<size_t>(j) * l + j] = 1.0 / R[static_cast<size_t>(j) * l + j];
    for (int i = j - 1; i >= 0; --i) {
      cdv s(0, 0);
      for (int p = i + 1; p <= j; ++p) s += R[static_cast<size_t>(p) * l + i] * X[static_cast<size_t>(j) * l + p];
      X[static_cast<size_t>(j) * l + i] = -s / R[static_cast<size_t>(i) * l + i];
    }
  }
  return X;
}

// Orthonormalise the columns of the device matrix Q (rows x l) in place.
void orthonormalize(Dev& d, double2* Q, int rows, int l, double2* G_d, double2* R_d, double2* tmp, uint64_t& seed) {
  for (int pass = 0; pass < 2; ++pass) {
    d.gemm(l, l, rows, Q, rows, true, Q, rows, false, G_d, l);
    std::vector<cdv> G(static_cast<size_t>(l) * l), R;
    d.down(reinterpret_cast<double2*>(G.data()), G_d, G.size());
    if (cholesky_upper(l, G, R)) {
      const std::vector<cdv> Ri = upper_inverse(l, R);
      d.up(R_d, reinterpret_cast<const double2*>(Ri.data()), Ri.size());
      d.gemm(rows, l, l, Q, rows, false, R_d, l, false, tmp, rows);
      check_cuda(cudaMemcpyAsync(Q, tmp, sizeof(double2) * rows * l, cudaMemcpyDeviceToDevice, d.st), "copy Q");
      continue;
    }
    // Rank-deficient block: modified Gram-Schmidt on the host, replacing a
    // dependent column by a fresh random direction.
    std::vector<cdv> q(static_cast<size_t>(rows) * l);
    d.down(reinterpret_cast<double2*>(q.data()), Q, q.size());
    for (int j = 0; j < l; ++j) {
      cdv* v = &q[static_cast<size_t>(j) * rows];
      for (int attempt = 0;; ++attempt) {
        double n0 = 0;
        for (int i = 0; i < rows; ++i) n0 += std::norm(v[i]);
        for (int rep = 0; rep < 2; ++rep)
          for (int p = 0; p < j; ++p) {
            const cdv* u = &q[static_cast<size_t>(p) * rows];
            cdv s(0, 0);
            for (int i = 0; i < rows; ++i) s += std::conj(u[i]) * v[i];
            for (int i = 0; i < rows; ++i) v[i] -= s * u[i];
          }
        double nn = 0;
        for (int i = 0; i < rows; ++i) nn += std::norm(v[i]);
        nn = std::sqrt(nn);
        if (nn > 1e-10 * std::sqrt(std::max(n0, 1e-300)) && nn > 0) {
          for (int i = 0; i < rows; ++i) v[i] /= nn;
          break;
        }
        if (attempt >= 8) throw Error(HUV_ERR_TCC_DECOMPOSITION, "orthonormalisation: no independent direction");
        for (int i = 0; i < rows; ++i) {
          seed = seed * 6364136223846793005ull + 1442695040888963407ull;
          const double a = static_cast<double>(seed >> 11) / 9007199254740992.0 - 0.5;
          seed = seed * 6364136223846793005ull + 1442695040888963407ull;
          const double b = static_cast<double>(seed >> 11) / 9007199254740992.0 - 0.5;
          v[i] = cdv(a, b);
        }
      }
    }
    d.up(Q, reinterpret_cast<const double2*>(q.data()), q.size());
    return;
  }
}

}  // namespace

KernelSet build_kernels_device(const std::vector<SourcePoint>& points, const Optics& optics, int n, double pixel_nm,
                               double lambda, int max_kernels, double fraction, double defocus_nm, int device,
                               bool reference_rule) {
  const double df = 1.0 / (n * pixel_nm);
  const double cutoff = optics.cutoff(lambda);
  if (!(std::isfinite(cutoff) && cutoff > 0.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "cutoff_frequency: optics cutoff NA/lambda must be positive");
  double sigma_max = 0.0;
  for (const auto& p : points) sigma_max = std::max(sigma_max, std::hypot(p.sx, p.sy));
  const double radius = cutoff * (1.0 + sigma_max);
  const double r2 = (radius / df) * (radius / df) * (1.0 + 1e-12);
  KernelSet ks;
  ks.n = n;
  ks.exceeds_nyquist = radius > (n / 2) * df;
  ks.defocus_nm = defocus_nm;
  ks.wavelength_nm = lambda;
  // Candidate orders in the same order as the host build.
  std::vector<int64_t> cidx;
  std::vector<double2> cand;
  for (int i = 0; i < n; ++i) {
    const double ky = i < n / 2 ? i : i - n;
    if (ky * ky > r2) continue;
    for (int j = 0; j < n; ++j) {
      const double kx = j < n / 2 ? j : j - n;
      if (kx * kx + ky * ky <= r2) {
        cidx.push_back(static_cast<int64_t>(i) * n + j);
        cand.push_back(make_double2(kx * df / cutoff, ky * df / cutoff));
      }
    }
  }
  const int64_t n_cand = static_cast<int64_t>(cand.size());
  const int64_t n_pts = static_cast<int64_t>(points.size());
  if (n_cand == 0 || n_pts == 0) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  if (n_cand * n_pts * 16 > (int64_t(1) << 30))
    throw Error(HUV_ERR_PUPIL_SAMPLING_TOO_DENSE,
                "pupil sampling too dense: the TCC factor would exceed 1 GiB; use a coarser grid");
  // Which entries are non-zero is decided by the pupil's support alone
  // (|rho| <= 1, rho >= obscuration, non-zero transmission): boolean tests on
  // the host, the complex values on the device.
  const double amp = optics.kind == HUV_OPTICS_EUV ? std::sqrt(std::max(optics.transmission, 0.0)) : 1.0;
  auto supported = [&](int64_t r, int64_t c) {
    const double fx = cand[r].x + points[c].sx, fy = cand[r].y + points[c].sy;
    const double rho2 = fx * fx + fy * fy;
    if (rho2 > 1.0 || amp == 0.0) return false;
    if (optics.kind == HUV_OPTICS_EUV && std::sqrt(rho2) < optics.obscuration) return false;
    return true;
  };
  std::vector<int64_t> keep_cols;
  std::vector<char> row_used(n_cand, 0);
  double clear = 0.0;
  for (int64_t c = 0; c < n_pts; ++c) {
    bool nz = false;
    for (int64_t r = 0; r < n_cand; ++r)
      if (supported(r, c)) {
        nz = true;
        row_used[r] = 1;
      }
    if (nz) keep_cols.push_back(c);
    if (supported(0, c)) clear += points[c].w * amp * amp;
  }
  const int64_t n_eff = static_cast<int64_t>(keep_cols.size());
  if (n_eff == 0) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  ks.clear_field = clear;
  ks.pupil_peak = amp * amp;
  ks.num_columns = static_cast<int>(n_eff);
  // Method: the reference's rule (aerial.rs:1116-1128) or always dense.
  const int64_t min_dim = std::min(n_cand, n_eff);
  const int64_t subspace = static_cast<int64_t>(max_kernels) + 16;
  const bool dense = !reference_rule || min_dim <= 320 || (min_dim <= 1536 && subspace * 3 >= min_dim);
  const int method = !dense ? 2 : (n_cand <= n_pts ? 0 : 1);
  ks.method = method;

  huv::Dev d(device);
  // A over the kept columns (column-major n_cand x n_eff).
  std::vector<double3> pts(n_eff);
  for (int64_t c = 0; c < n_eff; ++c)
    pts[c] = make_double3(points[keep_cols[c]].sx, points[keep_cols[c]].sy, points[keep_cols[c]].w);
  double2* cand_d = d.alloc<double2>(n_cand);
  double3* pts_d = d.alloc<double3>(n_eff);
  double2* A = d.alloc<double2>(static_cast<size_t>(n_cand * n_eff));
  d.up(cand_d, cand.data(), cand.size());
  d.up(pts_d, pts.data(), pts.size());
  huv_dev::DevOptics o{optics.kind, optics.na, optics.medium, optics.obscuration, amp, optics.paraxial ? 1 : 0};
  huv_dev::kb_fill_a<<<1184, 256, 0, d.st>>>(o, cand_d, pts_d, static_cast<int>(n_cand), static_cast<int>(n_eff),
                                               defocus_nm, lambda, A);
  check_cuda(cudaGetLastError(), "kb_fill_a");
  // trace = ||A||_F^2 = sum_s w_s |P|^2 over supported entries (host, exact)
  double trace = 0.0;
  for (int64_t c = 0; c < n_eff; ++c)
    for (int64_t r = 0; r < n_cand; ++r)
      if (supported(r, keep_cols[c])) trace += points[keep_cols[c]].w * amp * amp;

  if (method == 0) {
    std::vector<int64_t> rows;
    for (int64_t r = 0; r < n_cand; ++r)
      if (row_used[r]) rows.push_back(r);
    const int64_t m = static_cast<int64_t>(rows.size());
    // TCC over all candidates, then the used rows/columns on the host.
    double2* H = d.alloc<double2>(static_cast<size_t>(n_cand * n_cand));
    d.gemm(static_cast<int>(n_cand), static_cast<int>(n_cand), static_cast<int>(n_eff), A,
           static_cast<int>(n_cand), false, A, static_cast<int>(n_cand), true, H, static_cast<int>(n_cand));
    std::vector<cd> hf(static_cast<size_t>(n_cand * n_cand));
    d.down(reinterpret_cast<double2*>(hf.data()), H, hf.size());
    std::vector<cd> tcc(static_cast<size_t>(m * m));
    for (int64_t j = 0; j < m; ++j)
      for (int64_t i = 0; i < m; ++i) tcc[static_cast<size_t>(j * m + i)] = hf[static_cast<size_t>(rows[j] * n_cand + rows[i])];
    std::vector<double> vals;
    std::vector<cd> vecs;
    hermitian_eigen(static_cast<int>(m), tcc, vals, vecs, static_cast<int>(std::min<int64_t>(m, max_kernels)));
    const int k = select_kernel_count(vals, trace, max_kernels, fraction);
    ks.trace = trace;
    ks.eigenvalues.assign(vals.begin(), vals.begin() + k);
    ks.all_values = vals;
    ks.values.assign(vecs.begin(), vecs.begin() + static_cast<size_t>(k) * m);
    ks.support.resize(m);
    for (int64_t i = 0; i < m; ++i) ks.support[i] = cidx[rows[i]];
  } else if (method == 1) {
    double2* G = d.alloc<double2>(static_cast<size_t>(n_eff * n_eff));
    d.gemm(static_cast<int>(n_eff), static_cast<int>(n_eff), static_cast<int>(n_cand), A, static_cast<int>(n_cand),
           true, A, static_cast<int>(n_cand), false, G, static_cast<int>(n_eff));
    std::vector<cd> g(static_cast<size_t>(n_eff * n_eff));
    d.down(reinterpret_cast<double2*>(g.data()), G, g.size());
    std::vector<double> vals;
    std::vector<cd> vecs;
    hermitian_eigen(static_cast<int>(n_eff), g, vals, vecs, static_cast<int>(std::min<int64_t>(n_eff, max_kernels)));
    const int k = select_kernel_count(vals, trace, max_kernels, fraction);
    ks.trace = trace;
    ks.eigenvalues.assign(vals.begin(), vals.begin() + k);
    ks.all_values = vals;
    // u_k = A v_k / sqrt(lambda_k) on the device.
    double2* V = d.alloc<double2>(static_cast<size_t>(n_eff * k));
    double2* U = d.alloc<double2>(static_cast<size_t>(n_cand * k));
    double* s = d.alloc<double>(k);
    std::vector<double> inv(k);
    for (int q = 0; q < k; ++q) inv[q] = 1.0 / std::sqrt(ks.eigenvalues[q]);
    d.up(V, reinterpret_cast<const double2*>(vecs.data()), static_cast<size_t>(n_eff * k));
    d.up(s, inv.data(), inv.size());
    d.gemm(static_cast<int>(n_cand), k, static_cast<int>(n_eff), A, static_cast<int>(n_cand), false, V,
           static_cast<int>(n_eff), false, U, static_cast<int>(n_cand));
    huv_dev::kb_scale_cols<<<256, 256, 0, d.st>>>(U, static_cast<int>(n_cand), k, s);
    check_cuda(cudaGetLastError(), "kb_scale_cols");
    ks.values.resize(static_cast<size_t>(k) * n_cand);
    d.down(reinterpret_cast<double2*>(ks.values.data()), U, ks.values.size());
    ks.support = cidx;
  } else {
    const int l = static_cast<int>(std::min<int64_t>(subspace, min_dim));
    const int rows = static_cast<int>(n_cand), cols = static_cast<int>(n_eff);
    double2* Om = d.alloc<double2>(static_cast<size_t>(cols) * l);
    double2* Q = d.alloc<double2>(static_cast<size_t>(rows) * l);
    double2* Z = d.alloc<double2>(static_cast<size_t>(cols) * l);
    double2* tq = d.alloc<double2>(static_cast<size_t>(std::max(rows, cols)) * l);
    double2* G = d.alloc<double2>(static_cast<size_t>(l) * l);
    double2* R = d.alloc<double2>(static_cast<size_t>(l) * l);
    uint64_t seed = 0x5EED5EEDull;
    huv_dev::kb_gaussian<<<256, 256, 0, d.st>>>(Om, static_cast<size_t>(cols) * l, seed);
    check_cuda(cudaGetLastError(), "kb_gaussian");
    d.gemm(rows, l, cols, A, rows, false, Om, cols, false, Q, rows);
    orthonormalize(d, Q, rows, l, G, R, tq, seed);
    for (int it = 0; it < 3; ++it) {
      d.gemm(cols, l, rows, A, rows, true, Q, rows, false, Z, cols);
      orthonormalize(d, Z, cols, l, G, R, tq, seed);
      d.gemm(rows, l, cols, A, rows, false, Z, cols, false, Q, rows);
      orthonormalize(d, Q, rows, l, G, R, tq, seed);
    }
    d.gemm(cols, l, rows, A, rows, true, Q, rows, false, Z, cols);
    d.gemm(l, l, cols, Z, cols, true, Z, cols, false, G, l);
    std::vector<cd> t(static_cast<size_t>(l) * l);
    d.down(reinterpret_cast<double2*>(t.data()), G, t.size());
    std::vector<double> vals;
    std::vector<cd> w;
    hermitian_eigen(l, t, vals, w, l);
    const int k = select_kernel_count(vals, trace, std::min(max_kernels, l), fraction);
    ks.trace = trace;
    ks.eigenvalues.assign(vals.begin(), vals.begin() + k);
    ks.all_values = vals;
    double2* W = d.alloc<double2>(static_cast<size_t>(l) * k);
    double2* U = d.alloc<double2>(static_cast<size_t>(rows) * k);
    d.up(W, reinterpret_cast<const double2*>(w.data()), static_cast<size_t>(l) * k);
    d.gemm(rows, k, l, Q, rows, false, W, l, false, U, rows);
    ks.values.resize(static_cast<size_t>(k) * rows);
    d.down(reinterpret_cast<double2*>(ks.values.data()), U, ks.values.size());
    ks.support = cidx;
  }
  if (ks.eigenvalues.empty() || !(ks.trace > 0.0))
    throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  return ks;
}

}  // namespace huv
