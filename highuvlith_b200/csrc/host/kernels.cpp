// FP64 SOCS kernel build on the host: candidate mask orders, the exactly
// factorised TCC = A A^H with A[f, s] = sqrt(w_s) P((f + s) / f_c), a dense
// Hermitian eigensolve (TCC when the support is the smaller side, Gram A^H A
// otherwise), truncation on the eigenvalue tail.
//
// Follows KernelBuilder::build (crates/highuvlith-core/src/aerial.rs:1041-1317)
// and select_kernel_count (aerial.rs:992-1029).  The reference switches to a
// randomized eigensolver for large problems; the host builder always solves
// densely (exact), which the reference's own tests bound to 1e-5 in the image.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "host.hpp"

namespace huv {

// ----------------------------------------------------------- threading
int host_threads() {
  static int n = [] {
    const char* env = std::getenv("HUV_HOST_THREADS");
    int v = env ? std::atoi(env) : 0;
    if (v <= 0) v = static_cast<int>(std::thread::hardware_concurrency());
    return std::max(v, 1);
  }();
  return n;
}

namespace {
// Persistent worker pool: parallel_for is called thousands of times per
// eigensolve (twice per Householder step), so threads are started once.
// A parallel_for issued from inside a worker runs serially.
class Pool {
 public:
  explicit Pool(int n) {
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> l(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  int size() const { return static_cast<int>(workers_.size()); }
  // Runs body(b, e) over chunks of [0, n); the caller works too.  Returns
  // once every chunk has run and no worker is inside the region.
  void run(int64_t n, int chunks, const std::function<void(int64_t, int64_t)>& body) {
    std::lock_guard<std::mutex> region(run_mu_);
    const int64_t chunk = (n + chunks - 1) / chunks;
    {
      std::lock_guard<std::mutex> g(mu_);
      body_ = &body;
      n_ = n;
      chunk_ = chunk;
      next_.store(0);
      pending_ = (n + chunk - 1) / chunk;
      ++generation_;
    }
    cv_.notify_all();
    work(body, n, chunk);
    std::unique_lock<std::mutex> g(mu_);
    done_cv_.wait(g, [this] { return pending_ == 0 && active_ == 0; });
    body_ = nullptr;
  }
  static bool& in_worker() {
    static thread_local bool w = false;
    return w;
  }

 private:
  void work(const std::function<void(int64_t, int64_t)>& body, int64_t n, int64_t chunk) {
    for (;;) {
      const int64_t b = next_.fetch_add(1) * chunk;
      if (b >= n) break;
      body(b, std::min(n, b + chunk));
      std::lock_guard<std::mutex> g(mu_);
      if (--pending_ == 0) done_cv_.notify_all();
    }
  }
  void loop() {
    in_worker() = true;
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int64_t, int64_t)>* body;
      int64_t n, chunk;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || (generation_ != seen && body_ != nullptr); });
        if (stop_) return;
        seen = generation_;
        body = body_;
        n = n_;
        chunk = chunk_;
        ++active_;
      }
      work(*body, n, chunk);
      std::lock_guard<std::mutex> g(mu_);
      if (--active_ == 0 && pending_ == 0) done_cv_.notify_all();
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int64_t, int64_t)>* body_ = nullptr;
  int64_t n_ = 0, chunk_ = 1;
  std::atomic<int64_t> next_{0};
  int64_t pending_ = 0;
  int active_ = 0;
  uint64_t generation_ = 0;
  bool stop_ = false;
};

Pool& pool() {
  static Pool p(std::max(host_threads() - 1, 0));
  return p;
}
}  // namespace

SerialHostScope::SerialHostScope() : prev(Pool::in_worker()) { Pool::in_worker() = true; }
SerialHostScope::~SerialHostScope() { Pool::in_worker() = prev; }

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& body) {
  const int t = static_cast<int>(std::min<int64_t>(host_threads(), std::max<int64_t>(n / 64, 1)));
  if (t <= 1 || n < 128 || Pool::in_worker()) {
    body(0, n);
    return;
  }
  Pool& p = pool();
  if (p.size() == 0) {
    body(0, n);
    return;
  }
  p.run(n, t, body);
}

// ----------------------------------------------------------- selection
int select_kernel_count(const std::vector<double>& values, double trace, int max_kernels,
                        double fraction) {
  if (values.empty()) return 0;
  const double lead = values[0];
  if (std::isnan(lead) || lead <= 0.0) return 0;
  const double tol = 1e-12 * lead;
  int n_valid = 0;
  while (n_valid < static_cast<int>(values.size()) && values[n_valid] > tol) ++n_valid;
  const int cap = std::min(max_kernels, n_valid);
  int k = cap;
  if (fraction < 1.0) {
    double acc = 0.0;
    for (int i = 0; i < cap; ++i) {
      acc += values[i];
      if (acc >= fraction * trace) {
        k = i + 1;
        break;
      }
    }
  }
  auto same = [](double a, double b) {
    return std::fabs(a - b) <= 1e-6 * std::max(std::fabs(a), std::fabs(b));
  };
  if (k > 0 && k < n_valid && same(values[k - 1], values[k])) {
    int end = k;
    while (end < n_valid && same(values[end - 1], values[end])) ++end;
    if (end <= max_kernels) {
      k = end;
    } else {
      while (k > 0 && same(values[k - 1], values[k])) --k;
      if (k == 0) k = end;
    }
  }
  return k;
}

// ----------------------------------------------------------- eigensolver
namespace {

// Hermitian eigendecomposition by Householder reduction to a real symmetric
// tridiagonal (after a diagonal phase change), implicit QL with Wilkinson
// shifts accumulating the tridiagonal's eigenvectors, and a back-transform
// of only the requested eigenvectors.
class HermitianEigen {
 public:
  explicit HermitianEigen(int n, std::vector<cd> a) : n_(n) { decompose(std::move(a)); }
  const std::vector<double>& values() const { return values_; }
  std::vector<cd> vectors(int count) const;

 private:
  void decompose(std::vector<cd> a);
  std::vector<double> tridiag_vectors(int count) const;
  int n_;
  double scale_ = 1.0;
  std::vector<double> values_;
  std::vector<std::vector<cd>> refl_;  // unit Householder vectors acting on rows k+1..n-1
  std::vector<cd> phase_;
  std::vector<double> td_, te_;        // the real tridiagonal (scaled): diagonal, off-diagonal
  std::vector<double> tvals_;          // its eigenvalues, decreasing (scaled)
};

// Implicit symmetric QL on (d, e); e[i] couples d[i], d[i+1].  Accumulates
// rotations into z (column-major n x n) unless z is empty (eigenvalues only).
bool tridiag_ql(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z) {
  const bool vecs = !z.empty();
  if (n == 0) return true;
  double dmax = 0, emax = 0;
  for (int i = 0; i < n; ++i) dmax = std::max(dmax, std::fabs(d[i]));
  for (int i = 0; i < n; ++i) emax = std::max(emax, std::fabs(e[i]));
  const double eps = std::numeric_limits<double>::epsilon();
  const double floor_tol = eps * (dmax + 2.0 * emax);
  for (int l = 0; l < n; ++l) {
    for (int iter = 0;; ++iter) {
      int m = l;
      for (; m + 1 < n; ++m) {
        const double scale = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * scale || std::fabs(e[m]) <= floor_tol) break;
      }
      if (m == l) break;
      if (iter >= 120) return false;
      // Wilkinson-type shift from the 2x2 block at l.
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool early = false;
      for (int i = m - 1; i >= l; --i) {
        double f = s * e[i];
        const double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          early = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        if (vecs) {
          double* zi = &z[static_cast<size_t>(i) * n];
          double* zj = &z[static_cast<size_t>(i + 1) * n];
          for (int q = 0; q < n; ++q) {
            const double t = zj[q];
            zj[q] = s * zi[q] + c * t;
            zi[q] = c * zi[q] - s * t;
          }
        }
      }
      if (early) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

void HermitianEigen::decompose(std::vector<cd> a) {
  const int n = n_;
  double scale = 0.0;
  for (const cd& v : a) scale = std::max(scale, std::abs(v));
  const double inv = scale > 0 ? 1.0 / scale : 1.0;
  for (cd& v : a) v *= inv;
  auto A = [&](int i, int j) -> cd& { return a[static_cast<size_t>(j) * n + i]; };
  std::vector<cd> sub(std::max(n - 1, 0), cd(0, 0));
  refl_.assign(std::max(n - 2, 0), {});
  std::vector<cd> u, p;
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    double alpha2 = 0.0;
    for (int i = 0; i < m; ++i) alpha2 += std::norm(A(k + 1 + i, k));
    const double alpha = std::sqrt(alpha2);
    if (alpha == 0.0) continue;
    const cd x0 = A(k + 1, k);
    const cd ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : cd(1, 0);
    const cd beta = -ph * alpha;
    u.assign(m, cd(0, 0));
    for (int i = 0; i < m; ++i) u[i] = A(k + 1 + i, k);
    u[0] -= beta;
    double un = 0;
    for (const cd& v : u) un += std::norm(v);
    un = std::sqrt(un);
    for (cd& v : u) v /= un;
    // p = 2 A22 u ; K = u^H p ; q = p - K u ; A22 -= u q^H + q u^H
    p.assign(m, cd(0, 0));
    parallel_for(m, [&](int64_t b, int64_t e2) {
      for (int64_t i = b; i < e2; ++i) {
        // (A22 u)_i = sum_j A[i][j] u_j = sum_j conj(A[j][i]) u_j; column i is contiguous.
        const double* col = reinterpret_cast<const double*>(&a[static_cast<size_t>(k + 1 + i) * n + (k + 1)]);
        const double* uu = reinterpret_cast<const double*>(u.data());
        double re = 0.0, im = 0.0;
        for (int j = 0; j < m; ++j) {
          re += col[2 * j] * uu[2 * j] + col[2 * j + 1] * uu[2 * j + 1];
          im += col[2 * j] * uu[2 * j + 1] - col[2 * j + 1] * uu[2 * j];
        }
        p[i] = cd(2.0 * re, 2.0 * im);
      }
    });
    cd kk(0, 0);
    for (int i = 0; i < m; ++i) kk += std::conj(u[i]) * p[i];
    const double kr = kk.real();
    for (int i = 0; i < m; ++i) p[i] -= kr * u[i];
    parallel_for(m, [&](int64_t b, int64_t e2) {
      for (int64_t j = b; j < e2; ++j) {
        // col -= u conj(p_j) + p conj(u_j)
        const double qr = p[j].real(), qi = -p[j].imag(), vr = u[j].real(), vi = -u[j].imag();
        double* col = reinterpret_cast<double*>(&a[static_cast<size_t>(k + 1 + j) * n + (k + 1)]);
        const double* uu = reinterpret_cast<const double*>(u.data());
        const double* pp = reinterpret_cast<const double*>(p.data());
        for (int i = 0; i < m; ++i) {
          const double ur = uu[2 * i], ui = uu[2 * i + 1], pr = pp[2 * i], pi = pp[2 * i + 1];
          col[2 * i] -= ur * qr - ui * qi + pr * vr - pi * vi;
          col[2 * i + 1] -= ur * qi + ui * qr + pr * vi + pi * vr;
        }
      }
    });
    sub[k] = beta;
    refl_[k] = u;
  }
  if (n >= 2) sub[n - 2] = A(n - 1, n - 2);
  std::vector<double> d(n), e(n, 0.0);
  for (int i = 0; i < n; ++i) d[i] = A(i, i).real();
  for (int i = 0; i + 1 < n; ++i) e[i] = std::abs(sub[i]);
  phase_.assign(n, cd(1, 0));
  for (int k = 0; k + 1 < n; ++k) {
    const double r = std::abs(sub[k]);
    phase_[k + 1] = r > 0 ? phase_[k] * (sub[k] / r) : phase_[k];
  }
  td_ = d;
  te_ = e;
  // Eigenvalues by implicit QL without vectors (O(n^2)); eigenvectors are
  // computed on demand for the retained kernels only (tridiag_vectors).
  std::vector<double> none;
  if (!tridiag_ql(n, d, e, none))
    throw Error(HUV_ERR_TCC_DECOMPOSITION, "Hermitian eigensolver: QL iteration did not converge");
  std::sort(d.begin(), d.end(), [](double x, double y) { return x > y; });
  tvals_ = d;
  scale_ = scale;
  values_.resize(n);
  for (int i = 0; i < n; ++i) values_[i] = d[i] * scale;
}

// Eigenvectors of the real symmetric tridiagonal (td_, te_) for its `count`
// largest eigenvalues, by inverse iteration: LU with partial pivoting of
// T - lambda I (the tridiagonal form of LAPACK's gttrf/gttrs), three solves
// from a fixed start vector, each followed by modified Gram-Schmidt against
// the vectors already found for eigenvalues within 1e-3 ||T|| (a cluster:
// equal eigenvalues get an orthonormal basis of their eigenspace).  Returns
// column-major n x count.
std::vector<double> HermitianEigen::tridiag_vectors(int count) const {
  const int n = n_;
  std::vector<double> z(static_cast<size_t>(n) * count, 0.0);
  if (n == 1) {
    for (int c = 0; c < count; ++c) z[c] = 1.0;
    return z;
  }
  double tnorm = 0.0;
  for (int i = 0; i < n; ++i)
    tnorm = std::max(tnorm, std::fabs(td_[i]) + (i > 0 ? std::fabs(te_[i - 1]) : 0.0) + std::fabs(te_[i]));
  if (tnorm == 0.0) tnorm = 1.0;
  const double eps = std::numeric_limits<double>::epsilon();
  const double pivmin = eps * tnorm;
  const double ortol = 1e-3 * tnorm;
  std::vector<double> dl(n), dd(n), du(n), du2(n), x(n);
  std::vector<int> ipiv(n);
  int cluster_start = 0;
  double lam_prev = 0.0;
  for (int c = 0; c < count; ++c) {
    double lam = tvals_[c];
    if (c > 0 && lam_prev - lam > ortol) cluster_start = c;
    // separate equal eigenvalues slightly so each solve stays well posed
    if (c > cluster_start && lam >= lam_prev - 10.0 * eps * tnorm) lam = lam_prev - 10.0 * eps * tnorm;
    lam_prev = lam;
    // LU of T - lam I with partial pivoting
    for (int i = 0; i < n; ++i) dd[i] = td_[i] - lam;
    for (int i = 0; i + 1 < n; ++i) {
      dl[i] = te_[i];
      du[i] = te_[i];
    }
    for (int i = 0; i + 1 < n; ++i) {
      if (std::fabs(dd[i]) >= std::fabs(dl[i])) {
        if (dd[i] == 0.0) dd[i] = pivmin;
        const double f = dl[i] / dd[i];
        dl[i] = f;
        dd[i + 1] -= f * du[i];
        du2[i] = 0.0;
        ipiv[i] = i;
      } else {
        const double f = dd[i] / dl[i];
        dd[i] = dl[i];
        dl[i] = f;
        const double t = du[i];
        du[i] = dd[i + 1];
        dd[i + 1] = t - f * dd[i + 1];
        if (i + 2 < n) {
          du2[i] = du[i + 1];
          du[i + 1] = -f * du[i + 1];
        } else {
          du2[i] = 0.0;
        }
        ipiv[i] = i + 1;
      }
    }
    if (dd[n - 1] == 0.0) dd[n - 1] = pivmin;
    // fixed, non-degenerate start vector
    for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.5 * std::sin(1.0 + 0.7 * i + 0.37 * c);
    for (int it = 0; it < 3; ++it) {
      for (int i = 0; i + 1 < n; ++i) {
        if (ipiv[i] == i) {
          x[i + 1] -= dl[i] * x[i];
        } else {
          const double t = x[i];
          x[i] = x[i + 1];
          x[i + 1] = t - dl[i] * x[i];
        }
      }
      x[n - 1] /= dd[n - 1];
      x[n - 2] = (x[n - 2] - du[n - 2] * x[n - 1]) / dd[n - 2];
      for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - du[i] * x[i + 1] - du2[i] * x[i + 2]) / dd[i];
      for (int q = cluster_start; q < c; ++q) {
        const double* zq = &z[static_cast<size_t>(q) * n];
        double dot = 0.0;
        for (int i = 0; i < n; ++i) dot += zq[i] * x[i];
        for (int i = 0; i < n; ++i) x[i] -= dot * zq[i];
      }
      double nrm = 0.0;
      for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
      nrm = std::sqrt(nrm);
      if (!(nrm > 0.0) || !std::isfinite(nrm))
        throw Error(HUV_ERR_TCC_DECOMPOSITION, "Hermitian eigensolver: inverse iteration broke down");
      for (int i = 0; i < n; ++i) x[i] /= nrm;
    }
    std::copy(x.begin(), x.end(), z.begin() + static_cast<size_t>(c) * n);
  }
  return z;
}

std::vector<cd> HermitianEigen::vectors(int count) const {
  const int n = n_;
  count = std::min(count, n);
  const std::vector<double> z = tridiag_vectors(count);
  std::vector<cd> w(static_cast<size_t>(n) * count);
  for (int c = 0; c < count; ++c)
    for (int i = 0; i < n; ++i) w[static_cast<size_t>(c) * n + i] = phase_[i] * z[static_cast<size_t>(c) * n + i];
  for (int k = static_cast<int>(refl_.size()) - 1; k >= 0; --k) {
    const auto& u = refl_[k];
    if (u.empty()) continue;
    for (int c = 0; c < count; ++c) {
      cd* tail = &w[static_cast<size_t>(c) * n + k + 1];
      cd t(0, 0);
      for (size_t i = 0; i < u.size(); ++i) t += std::conj(u[i]) * tail[i];
      t *= 2.0;
      for (size_t i = 0; i < u.size(); ++i) tail[i] -= u[i] * t;
    }
  }
  return w;
}

}  // namespace

void hermitian_eigen(int n, const std::vector<cd>& h, std::vector<double>& values,
                     std::vector<cd>& vectors, int count) {
  HermitianEigen eig(n, h);
  values = eig.values();
  vectors = eig.vectors(count);
}

// ----------------------------------------------------------- kernel set
int KernelSet::band_half_width() const {
  int h = 0;
  for (int64_t idx : support) {
    const int i = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
    const int ky = i < n / 2 ? i : i - n, kx = j < n / 2 ? j : j - n;
    h = std::max(h, std::max(std::abs(kx), std::abs(ky)));
  }
  return h;
}

double KernelSet::divisor(int normalization) const {
  const bool bright = clear_field > 0.0 && clear_field >= 1e-2 * pupil_peak;
  return (normalization == 0 && bright) ? clear_field : 0.0;
}

KernelSet build_kernels(const std::vector<SourcePoint>& points, const Optics& optics, int n,
                        double pixel_nm, double lambda, int max_kernels, double fraction,
                        double defocus_nm, int force_method) {
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
  struct Cand {
    int64_t idx;
    double fx, fy;
  };
  std::vector<Cand> cand;
  for (int i = 0; i < n; ++i) {
    const double ky = i < n / 2 ? i : i - n;
    if (ky * ky > r2) continue;
    for (int j = 0; j < n; ++j) {
      const double kx = j < n / 2 ? j : j - n;
      if (kx * kx + ky * ky <= r2)
        cand.push_back(Cand{static_cast<int64_t>(i) * n + j, kx * df / cutoff, ky * df / cutoff});
    }
  }
  const int64_t n_cand = static_cast<int64_t>(cand.size());
  const int64_t n_pts = static_cast<int64_t>(points.size());
  if (n_cand == 0 || n_pts == 0) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  if (n_cand * n_pts * 16 > (int64_t(1) << 30))
    throw Error(HUV_ERR_PUPIL_SAMPLING_TOO_DENSE,
                "pupil sampling too dense: the TCC factor would exceed 1 GiB; use a coarser grid");
  // A, column-major n_cand x n_pts.
  std::vector<cd> a(static_cast<size_t>(n_cand * n_pts));
  parallel_for(n_pts, [&](int64_t b, int64_t e) {
    for (int64_t c = b; c < e; ++c) {
      const double amp = std::sqrt(points[c].w);
      cd* col = &a[static_cast<size_t>(c * n_cand)];
      for (int64_t r = 0; r < n_cand; ++r)
        col[r] = optics.pupil(cand[r].fx + points[c].sx, cand[r].fy + points[c].sy, defocus_nm, lambda) * amp;
    }
  });
  double clear = 0.0, peak = 0.0;
  for (int64_t c = 0; c < n_pts; ++c) clear += std::norm(a[static_cast<size_t>(c * n_cand)]);
  for (int64_t c = 0; c < n_pts; ++c) {
    const double w = points[c].w;
    for (int64_t r = 0; r < n_cand; ++r) peak = std::max(peak, std::norm(a[static_cast<size_t>(c * n_cand + r)]) / w);
  }
  ks.clear_field = clear;
  ks.pupil_peak = peak;
  // Drop all-zero columns.
  std::vector<int64_t> keep_cols;
  for (int64_t c = 0; c < n_pts; ++c) {
    bool nz = false;
    for (int64_t r = 0; r < n_cand && !nz; ++r) {
      const cd v = a[static_cast<size_t>(c * n_cand + r)];
      nz = v.real() != 0.0 || v.imag() != 0.0;
    }
    if (nz) keep_cols.push_back(c);
  }
  const int64_t n_eff = static_cast<int64_t>(keep_cols.size());
  if (n_eff == 0) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  ks.num_columns = static_cast<int>(n_eff);
  const int method = force_method >= 0 ? force_method : (n_cand <= n_pts ? 0 : 1);
  ks.method = method;
  if (method == 0) {
    // TCC over the support rows that any kept column reaches.
    std::vector<int64_t> rows;
    for (int64_t r = 0; r < n_cand; ++r) {
      bool nz = false;
      for (int64_t c : keep_cols) {
        const cd v = a[static_cast<size_t>(c * n_cand + r)];
        if (v.real() != 0.0 || v.imag() != 0.0) {
          nz = true;
          break;
        }
      }
      if (nz) rows.push_back(r);
    }
    const int64_t m = static_cast<int64_t>(rows.size());
    if (m == 0) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
    double trace = 0.0;
    for (int64_t r : rows)
      for (int64_t c : keep_cols) trace += std::norm(a[static_cast<size_t>(c * n_cand + r)]);
    // TCC[f, f'] = sum_s A[f, s] conj(A[f', s]), column-major m x m, from a
    // row-major copy of the used rows (contiguous dot products, one triangle).
    const int64_t nk = static_cast<int64_t>(keep_cols.size());
    std::vector<cd> yr(static_cast<size_t>(m * nk));
    parallel_for(m, [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i)
        for (int64_t c = 0; c < nk; ++c)
          yr[static_cast<size_t>(i * nk + c)] = a[static_cast<size_t>(keep_cols[c] * n_cand + rows[i])];
    });
    std::vector<cd> tcc(static_cast<size_t>(m * m));
    parallel_for(m, [&](int64_t b, int64_t e) {
      for (int64_t jj = b; jj < e; ++jj) {
        const cd* yj = &yr[static_cast<size_t>(jj * nk)];
        for (int64_t ii = jj; ii < m; ++ii) {
          const cd* yi = &yr[static_cast<size_t>(ii * nk)];
          double re = 0, im = 0;
          for (int64_t c = 0; c < nk; ++c) {
            // yi[c] * conj(yj[c])
            re += yi[c].real() * yj[c].real() + yi[c].imag() * yj[c].imag();
            im += yi[c].imag() * yj[c].real() - yi[c].real() * yj[c].imag();
          }
          tcc[static_cast<size_t>(jj * m + ii)] = cd(re, im);
          tcc[static_cast<size_t>(ii * m + jj)] = cd(re, -im);
        }
      }
    });
    HermitianEigen eig(static_cast<int>(m), std::move(tcc));
    const int k = select_kernel_count(eig.values(), trace, max_kernels, fraction);
    std::vector<cd> v = eig.vectors(k);
    ks.trace = trace;
    ks.eigenvalues.assign(eig.values().begin(), eig.values().begin() + k);
    ks.all_values = eig.values();
    ks.values = std::move(v);  // k x m, kernel-major (columns of V)
    ks.support.resize(m);
    for (int64_t i = 0; i < m; ++i) ks.support[i] = cand[rows[i]].idx;
  } else {
    double trace = 0.0;
    for (int64_t c : keep_cols)
      for (int64_t r = 0; r < n_cand; ++r) trace += std::norm(a[static_cast<size_t>(c * n_cand + r)]);
    // Gram G = A^H A over kept columns, column-major n_eff x n_eff.
    std::vector<cd> g(static_cast<size_t>(n_eff * n_eff));
    parallel_for(n_eff, [&](int64_t b, int64_t e) {
      for (int64_t j = b; j < e; ++j) {
        const cd* cj = &a[static_cast<size_t>(keep_cols[j] * n_cand)];
        for (int64_t i = 0; i <= j; ++i) {
          const cd* ci = &a[static_cast<size_t>(keep_cols[i] * n_cand)];
          double re = 0, im = 0;
          for (int64_t r = 0; r < n_cand; ++r) {
            // conj(ci[r]) * cj[r]
            re += ci[r].real() * cj[r].real() + ci[r].imag() * cj[r].imag();
            im += ci[r].real() * cj[r].imag() - ci[r].imag() * cj[r].real();
          }
          g[static_cast<size_t>(j * n_eff + i)] = cd(re, im);
          g[static_cast<size_t>(i * n_eff + j)] = cd(re, -im);
        }
      }
    });
    HermitianEigen eig(static_cast<int>(n_eff), std::move(g));
    const int k = select_kernel_count(eig.values(), trace, max_kernels, fraction);
    std::vector<cd> v = eig.vectors(k);
    ks.trace = trace;
    ks.eigenvalues.assign(eig.values().begin(), eig.values().begin() + k);
    ks.all_values = eig.values();
    // u_k = A v_k / sqrt(lambda_k) over every candidate (columns of A are
    // contiguous: accumulate column by column over a block of rows).
    ks.values.assign(static_cast<size_t>(k) * n_cand, cd(0, 0));
    parallel_for(n_cand, [&](int64_t b, int64_t e) {
      for (int q = 0; q < k; ++q) {
        cd* out = &ks.values[static_cast<size_t>(q * n_cand)];
        for (int64_t j = 0; j < n_eff; ++j) {
          const cd vj = v[static_cast<size_t>(q * n_eff + j)];
          const cd* col = &a[static_cast<size_t>(keep_cols[j] * n_cand)];
          for (int64_t r = b; r < e; ++r) out[r] += col[r] * vj;
        }
        const double inv = 1.0 / std::sqrt(ks.eigenvalues[q]);
        for (int64_t r = b; r < e; ++r) out[r] *= inv;
      }
    });
    ks.support.resize(n_cand);
    for (int64_t i = 0; i < n_cand; ++i) ks.support[i] = cand[i].idx;
  }
  if (ks.eigenvalues.empty() || !(ks.trace > 0.0))
    throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "no diffraction orders pass the pupil");
  return ks;
}

}  // namespace huv
