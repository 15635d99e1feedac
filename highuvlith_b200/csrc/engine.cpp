// Engine: FP64 host set-up + device kernel sets + the batched image pipeline,
// behind the C ABI of include/huv_b200.h.
//
// Mirrors AerialImageEngine (crates/highuvlith-core/src/aerial.rs:1472-1967):
// construction samples the source and builds the in-focus kernel set; other
// focus planes are built on demand and kept in a bounded LRU cache keyed by
// the focus plane (aerial.rs:1363-1464), with a device copy of each set.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine.hpp"

#include <atomic>
#include <exception>
#include <thread>
#include "host/host.hpp"

namespace huv_launch {
cudaError_t socs_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int lgm, int clips,
                      float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols(const float2* T, int K, int hb, int lgm, int clips, float keep, float flare,
                      const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
bool xt_ok(int L, int hb);
cudaError_t socs_rows_x(const float2* kband, float scale, const float2* Mband, int K, int hb, int L, int clips,
                        float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols_x(const float2* T, int K, int hb, int L, int clips, float keep, float flare,
                        const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
cudaError_t set_smem_limits();
bool field_fused_ok(int L, int hb);
size_t field_fused_part_bytes(int L, int K);
cudaError_t socs_field_fused(const float2* kband, const float2* Mband, int K, int hb, int L, int clips, float keep,
                             float flare, const float* mean, float* out, void* split, float* part, const float2* tw,
                             cudaStream_t st);
void tc_release(huv::TcState& tc);
void tc_release_all(std::map<int, huv::TcState>& m);
bool mask_rows_tc_supported(int n, int hb);
std::vector<uint8_t> mask_rows_tc_digits(int n, int hb);
}  // namespace huv_launch

namespace huv {

namespace {
thread_local std::string g_last_error = "";

inline int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
}  // namespace

void set_last_error(const std::string& m) { g_last_error = m; }
const char* last_error() { return g_last_error.c_str(); }

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation)
      throw Error(HUV_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    throw Error(HUV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// ------------------------------------------------------------ construction
Engine::Engine(const huv_source& s, const huv_optics& o, const huv_grid& g, const huv_settings& st,
               int dev)
    : settings(st), device(dev) {
  if (st.max_kernels < 1) throw Error(HUV_ERR_INVALID_PARAMETER, "max_kernels: must be at least 1");
  if (!(st.kernel_energy_fraction > 0.0 && st.kernel_energy_fraction <= 1.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "kernel_energy_fraction: must be in (0, 1]");
  if (st.source_points_per_axis < 0)
    throw Error(HUV_ERR_INVALID_PARAMETER, "source_points_per_axis: must be >= 0 (0 = adaptive)");
  if (g.size < 2 || !(std::isfinite(g.pixel_nm) && g.pixel_nm > 0.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "grid: needs size >= 2 and a positive finite pixel_nm");
  if ((g.size & (g.size - 1)) != 0)
    throw Error(HUV_ERR_GRID_NOT_POWER_OF_TWO, "grid size " + std::to_string(g.size) + " must be a power of 2");
  if (g.size < 8 || g.size > 8192)
    throw Error(HUV_ERR_UNSUPPORTED, "grid size must be in [8, 8192] for the device path");
  if (!(std::isfinite(s.wavelength_nm) && s.wavelength_nm > 0.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "wavelength_nm: must be positive and finite");
  if (s.fill < HUV_FILL_CONVENTIONAL || s.fill > HUV_FILL_QUASAR)
    throw Error(HUV_ERR_INVALID_PARAMETER, "illumination: unknown fill kind");
  fill.kind = s.fill;
  for (int i = 0; i < 4; ++i) fill.p[i] = s.p[i];
  fill.prepare();
  optics.kind = o.kind;
  optics.na = o.na;
  optics.flare = o.flare_fraction;
  optics.medium = o.kind == HUV_OPTICS_EUV ? 1.0 : (o.immersion_index > 0 ? o.immersion_index : 1.0);
  optics.obscuration = o.central_obscuration;
  optics.transmission = o.kind == HUV_OPTICS_EUV ? o.transmission : 1.0;
  optics.paraxial = o.paraxial_defocus != 0;
  if (!(std::isfinite(optics.medium) && optics.medium >= 1.0 && optics.na > 0.0 && optics.na < optics.medium))
    throw Error(HUV_ERR_INVALID_PARAMETER,
                "numerical_aperture: must be positive and below the image-space (immersion) index");
  if (o.kind == HUV_OPTICS_EUV && !(optics.obscuration >= 0.0 && optics.obscuration < 1.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "central_obscuration: must be in [0, 1)");
  if (!(optics.flare >= 0.0 && optics.flare < 1.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "flare_fraction: must be in [0, 1)");
  n = g.size;
  pixel_nm = g.pixel_nm;
  lambda = s.wavelength_nm;
  const double cutoff = optics.cutoff(lambda);
  const double df_sigma = (1.0 / (n * pixel_nm)) / cutoff;
  points = sample_source(fill, st.source_points_per_axis, df_sigma);
  if (st.kernel_build < HUV_BUILD_HOST || st.kernel_build > HUV_BUILD_DEVICE_RULE)
    throw Error(HUV_ERR_INVALID_PARAMETER, "kernel_build: unknown");
  focus = std::make_shared<KernelSet>(build_set(0.0));
}

Engine::Engine(const huv_kernel_set& set, int dev) : device(dev) {
  const int n_ = set.grid_size, K = set.n_kernels;
  if (n_ < 8 || n_ > 8192 || (n_ & (n_ - 1)) != 0)
    throw Error(HUV_ERR_GRID_NOT_POWER_OF_TWO, "kernel set: grid_size must be a power of two in [8, 8192]");
  if (K < 1) throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: n_kernels must be at least 1");
  if (!set.eigenvalues || !set.kernels) throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: null array");
  if (!(std::isfinite(set.defocus_nm))) throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: defocus_nm must be finite");
  if (!(set.flare_fraction >= 0.0 && set.flare_fraction < 1.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: flare_fraction must be in [0, 1)");
  if (!(set.captured_energy_fraction > 0.0 && set.captured_energy_fraction <= 1.0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: captured_energy_fraction must be in (0, 1]");
  for (int k = 0; k < K; ++k) {
    const double v = set.eigenvalues[k];
    if (!(std::isfinite(v) && v >= 0.0) || (k > 0 && v > set.eigenvalues[k - 1]))
      throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: eigenvalues must be finite, >= 0 and non-increasing");
  }
  n = n_;
  pixel_nm = std::isfinite(set.pixel_nm) && set.pixel_nm > 0 ? set.pixel_nm : 1.0;
  lambda = set.wavelength_nm;
  optics.flare = set.flare_fraction;
  fixed_set = true;
  fixed_z = set.defocus_nm;
  // images stay as the eigenvalues give them: the normalisation is folded in
  settings = huv_settings{K, 1.0, 0, 1, 0, HUV_BUILD_HOST};
  // sparse form: the union of the kernels' non-zero frequencies
  const size_t nn = static_cast<size_t>(n) * n;
  std::vector<char> used(nn, 0);
  for (int k = 0; k < K; ++k)
    for (size_t i = 0; i < nn; ++i) {
      const double re = set.kernels[2 * (k * nn + i)], im = set.kernels[2 * (k * nn + i) + 1];
      if (!(std::isfinite(re) && std::isfinite(im)))
        throw Error(HUV_ERR_INVALID_PARAMETER, "kernel set: kernels must be finite");
      if (re != 0.0 || im != 0.0) used[i] = 1;
    }
  auto ks = std::make_shared<KernelSet>();
  ks->n = n;
  for (size_t i = 0; i < nn; ++i)
    if (used[i]) ks->support.push_back(static_cast<int64_t>(i));
  if (ks->support.empty()) throw Error(HUV_ERR_NO_DIFFRACTION_ORDERS, "kernel set: every kernel is zero");
  const size_t S = ks->support.size();
  ks->values.resize(static_cast<size_t>(K) * S);
  for (int k = 0; k < K; ++k)
    for (size_t t = 0; t < S; ++t) {
      const size_t o = 2 * (k * nn + static_cast<size_t>(ks->support[t]));
      ks->values[k * S + t] = cd(set.kernels[o], set.kernels[o + 1]);
    }
  ks->eigenvalues.assign(set.eigenvalues, set.eigenvalues + K);
  ks->all_values = ks->eigenvalues;
  double sum = 0.0, clear = 0.0;
  for (int k = 0; k < K; ++k) {
    sum += ks->eigenvalues[k];
    // the field of a clear mask is the kernel's DC value (spectrum N^2 at DC, 1/N^2 inverse)
    if (ks->support[0] == 0) clear += ks->eigenvalues[k] * std::norm(ks->values[k * S]);
  }
  ks->trace = sum / set.captured_energy_fraction;
  ks->clear_field = clear;
  ks->pupil_peak = clear;
  ks->method = 3;  // supplied by the caller
  ks->num_columns = 0;
  ks->defocus_nm = set.defocus_nm;
  ks->wavelength_nm = set.wavelength_nm;
  ks->exceeds_nyquist = 2 * ks->band_half_width() >= n;
  focus = ks;
}

double Engine::plane_key(double z) const {
  if (!fixed_set) return z == 0.0 ? 0.0 : z;
  if (z == 0.0 || z == fixed_z) return 0.0;
  throw Error(HUV_ERR_UNSUPPORTED, "engine over a supplied kernel set: only its own focus plane (" +
                                       std::to_string(fixed_z) + " nm) can be imaged");
}

Engine::~Engine() {
  if (device_ready) {
    cudaSetDevice(device);
    for (auto& kv : twiddles) cudaFree(kv.second);
    for (auto& kv : row_digits) cudaFree(kv.second);
    auto free_set = [](DeviceSet& d) {
      for (auto& kv : d.W_by_k) cudaFree(kv.second);
      cudaFree(d.kband);
      cudaFree(d.W);
      cudaFree(d.ptx);
      huv_launch::tc_release_all(d.tc);
    };
    free_set(focus_dev);
    for (auto& e : cache) free_set(e.dev);
    prof.release();
    cudaFree(dev_err);
    cudaFree(ilt_cost_dev);
    ilt_state.release();
    cudaFree(ws);
    cudaFree(io_in);
    cudaFree(io_out);
    cudaFree(rect.clip_rows);
    cudaFree(rect.rows);
    cudaFree(rect.runs);
    cudaFree(rect.coef);
    if (io_h2d) {
      cudaStreamDestroy(io_h2d);
      cudaStreamDestroy(io_d2h);
      for (auto& row : io_ev)
        for (auto e : row) cudaEventDestroy(e);
    }
  }
}

KernelSet Engine::build_set(double z) {
  if (fixed_set) throw Error(HUV_ERR_UNSUPPORTED, "engine over a supplied kernel set: no other focus plane");
  if (settings.kernel_build == HUV_BUILD_HOST)
    return build_kernels(points, optics, n, pixel_nm, lambda, settings.max_kernels, settings.kernel_energy_fraction, z);
  return build_kernels_device(points, optics, n, pixel_nm, lambda, settings.max_kernels,
                              settings.kernel_energy_fraction, z, device,
                              settings.kernel_build == HUV_BUILD_DEVICE_RULE);
}

std::shared_ptr<KernelSet> Engine::kernel_set(double z) {
  z = plane_key(z);
  if (z == 0.0) return focus;
  for (auto& e : cache)
    if (e.z == z) {
      e.last_used = ++clock;
      return e.ks;
    }
  auto ks = std::make_shared<KernelSet>(build_set(z));
  cache_insert(z, ks);
  return ks;
}

std::shared_ptr<KernelSet> Engine::held_set(double z) {
  z = plane_key(z);
  if (z == 0.0) return focus;
  for (auto& e : cache)
    if (e.z == z) return e.ks;
  return nullptr;
}

void Engine::cache_insert(double z, std::shared_ptr<KernelSet> ks) {
  if (settings.kernel_cache_capacity <= 0) {
    scratch_set = ks;
    return;
  }
  if (static_cast<int>(cache.size()) >= settings.kernel_cache_capacity) {
    auto it = std::min_element(cache.begin(), cache.end(),
                               [](const CacheEntry& a, const CacheEntry& b) { return a.last_used < b.last_used; });
    if (device_ready) {
      for (auto& kv : it->dev.W_by_k) cudaFree(kv.second);
      cudaFree(it->dev.kband);
      cudaFree(it->dev.W);
      cudaFree(it->dev.ptx);
      huv_launch::tc_release_all(it->dev.tc);
    }
    cache.erase(it);
  }
  CacheEntry e;
  e.z = z;
  e.ks = ks;
  e.last_used = ++clock;
  cache.push_back(e);
}

void Engine::prebuild_planes(const double* z, int planes) {
  std::vector<double> todo;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (int p = 0; p < planes; ++p) {
      const double zz = plane_key(z[p]);
      if (zz == 0.0 || std::find(todo.begin(), todo.end(), zz) != todo.end()) continue;
      bool have = false;
      for (const auto& e : cache) have = have || e.z == zz;
      if (!have) todo.push_back(zz);
    }
    const size_t cap = static_cast<size_t>(std::max(settings.kernel_cache_capacity, 0));
    if (todo.size() > cap) todo.resize(cap);  // the rest is built on demand
  }
  if (todo.empty()) return;
  std::vector<std::shared_ptr<KernelSet>> built(todo.size());
  std::vector<std::exception_ptr> errs(todo.size());
  std::atomic<size_t> next{0};
  auto worker = [&] {
    SerialHostScope serial;
    for (size_t i; (i = next.fetch_add(1)) < todo.size();) {
      try {
        built[i] = std::make_shared<KernelSet>(build_set(todo[i]));
      } catch (...) {
        errs[i] = std::current_exception();
      }
    }
  };
  const int nt = static_cast<int>(std::min<size_t>(todo.size(), static_cast<size_t>(host_threads())));
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
  std::lock_guard<std::mutex> lock(mu);
  for (size_t i = 0; i < todo.size(); ++i) {
    bool have = false;
    for (const auto& e : cache) have = have || e.z == todo[i];
    if (!have) cache_insert(todo[i], built[i]);
  }
}

void Engine::image_focus_sweep(const huv_batch& b, const double* z, int planes, float* out, cudaStream_t st) {
  if (planes < 0) throw Error(HUV_ERR_INVALID_PARAMETER, "n_planes: must be >= 0");
  if (planes == 0 || b.n_clips == 0) return;
  if (!z || !out) throw Error(HUV_ERR_INVALID_PARAMETER, "focus/out: null pointer");
  for (int p = 0; p < planes; ++p)
    if (!std::isfinite(z[p])) throw Error(HUV_ERR_INVALID_PARAMETER, "focus_nm: must be finite");
  prebuild_planes(z, planes);
  const size_t plane = static_cast<size_t>(b.n_clips) * n * n;
  for (int p = 0; p < planes; ++p) {
    huv_batch bp = b;
    bp.defocus_nm = z[p];
    image_batch(bp, out + plane * p, st);
  }
}

// ------------------------------------------------------------ device side
void Engine::ensure_device() {
  check_cuda(cudaSetDevice(device), "cudaSetDevice");
  if (device_ready) return;
  check_cuda(huv_launch::set_smem_limits(), "cudaFuncSetAttribute");
  check_cuda(cudaMalloc(&dev_err, sizeof(int)), "cudaMalloc(error flag)");
  check_cuda(cudaMemset(dev_err, 0, sizeof(int)), "cudaMemset(error flag)");
  device_ready = true;
}

const float2* Engine::twiddle(int lg) { return twiddle_n(1 << lg); }

const float2* Engine::twiddle_n(int L) {
  auto it = twiddles.find(L);
  if (it != twiddles.end()) return it->second;
  std::vector<float2> h(L);
  for (int t = 0; t < L; ++t) {
    const double a = -2.0 * 3.14159265358979323846 * t / L;
    h[t] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  float2* d = nullptr;
  check_cuda(cudaMalloc(&d, sizeof(float2) * L), "cudaMalloc(twiddle)");
  check_cuda(cudaMemcpy(d, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice), "cudaMemcpy(twiddle)");
  twiddles[L] = d;
  return d;
}

const uint8_t* Engine::row_digit_table(int hb) {
  auto it = row_digits.find(hb);
  if (it != row_digits.end()) return it->second;
  const char* env = std::getenv("HUV_MASK_ROWS");
  uint8_t* d = nullptr;
  if (!(env && std::string(env) == "fft") && huv_launch::mask_rows_tc_supported(n, hb)) {
    const std::vector<uint8_t> h = huv_launch::mask_rows_tc_digits(n, hb);
    check_cuda(cudaMalloc(&d, h.size()), "cudaMalloc(row digits)");
    check_cuda(cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice), "cudaMemcpy(row digits)");
  }
  row_digits[hb] = d;
  return d;
}

DeviceSet& Engine::device_set(double z) {
  z = plane_key(z);
  std::shared_ptr<KernelSet> ks = kernel_set(z);
  DeviceSet* slot = nullptr;
  if (z == 0.0) {
    slot = &focus_dev;
  } else {
    for (auto& e : cache)
      if (e.z == z) slot = &e.dev;
    if (!slot) slot = &scratch_dev;
  }
  if (slot->kband && slot->source == ks.get()) return *slot;
  if (slot->kband) {
    for (auto& kv : slot->W_by_k) cudaFree(kv.second);
    cudaFree(slot->kband);
    cudaFree(slot->W);
    cudaFree(slot->ptx);
    huv_launch::tc_release_all(slot->tc);
    *slot = DeviceSet();
  }
  const int h = ks->band_half_width();
  const int B = 2 * h + 1;
  const int K = ks->num_kernels();
  const int S = static_cast<int>(ks->support.size());
  double div = ks->divisor(settings.normalization);
  if (div == 0.0) div = 1.0;
  const double n2 = static_cast<double>(n) * n;
  std::vector<float2> kb(static_cast<size_t>(K) * B * B, make_float2(0.f, 0.f));
  std::vector<double> wd(static_cast<size_t>(B) * B, 0.0);
  for (int k = 0; k < K; ++k) {
    const double lam = ks->eigenvalues[k] / div;
    const double sc = std::sqrt(lam) / n2;
    for (int t = 0; t < S; ++t) {
      const int64_t idx = ks->support[t];
      const int i = static_cast<int>(idx / n), j = static_cast<int>(idx % n);
      const int my = i < n / 2 ? i : i - n, mx = j < n / 2 ? j : j - n;
      const cd u = ks->values[static_cast<size_t>(k) * S + t];
      const size_t o = (static_cast<size_t>(my + h)) * B + (mx + h);
      kb[static_cast<size_t>(k) * B * B + o] = make_float2(static_cast<float>(u.real() * sc), static_cast<float>(u.imag() * sc));
      wd[o] += lam * std::norm(u) / (n2 * n2);
    }
  }
  std::vector<float> wf(wd.begin(), wd.end());
  std::vector<float> ptx(B);
  for (int i = 0; i < B; ++i) {
    const double u = 3.14159265358979323846 * (i - h) / n;
    ptx[i] = static_cast<float>(std::fabs(u) < 1e-6 ? 1.0 - u * u / 6.0 : std::sin(u) / u);
  }
  DeviceSet d;
  d.source = ks.get();
  d.hold = ks;
  d.hb = h;
  d.B = B;
  d.K = K;
  d.keep = optics.flare > 0.0 ? static_cast<float>(1.0 - optics.flare) : 1.f;
  d.flare = optics.flare > 0.0 ? static_cast<float>(optics.flare) : 0.f;
  d.eig_scaled.resize(K);
  for (int k = 0; k < K; ++k) d.eig_scaled[k] = ks->eigenvalues[k] / div;
  d.host_kband = kb;
  check_cuda(cudaMalloc(&d.kband, sizeof(float2) * kb.size()), "cudaMalloc(kband)");
  check_cuda(cudaMalloc(&d.W, sizeof(float) * wf.size()), "cudaMalloc(W)");
  check_cuda(cudaMalloc(&d.ptx, sizeof(float) * ptx.size()), "cudaMalloc(ptx)");
  check_cuda(cudaMemcpy(d.kband, kb.data(), sizeof(float2) * kb.size(), cudaMemcpyHostToDevice), "upload kband");
  check_cuda(cudaMemcpy(d.W, wf.data(), sizeof(float) * wf.size(), cudaMemcpyHostToDevice), "upload W");
  check_cuda(cudaMemcpy(d.ptx, ptx.data(), sizeof(float) * ptx.size(), cudaMemcpyHostToDevice), "upload ptx");
  *slot = std::move(d);
  return *slot;
}

const float* Engine::flare_weights(DeviceSet& ds, int K) {
  if (K <= 0 || K >= ds.K) return ds.W;
  auto it = ds.W_by_k.find(K);
  if (it != ds.W_by_k.end()) return it->second;
  const int B = ds.B;
  std::vector<float> w(static_cast<size_t>(B) * B, 0.f);
  std::vector<double> wd(static_cast<size_t>(B) * B, 0.0);
  for (int k = 0; k < K; ++k)
    for (size_t i = 0; i < wd.size(); ++i) {
      // |kappa_k|^2 = lambda_k |u_k|^2 / N^4 (the band kernels carry sqrt(lambda)/N^2)
      const float2 v = ds.host_kband[static_cast<size_t>(k) * B * B + i];
      wd[i] += static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
    }
  for (size_t i = 0; i < wd.size(); ++i) w[i] = static_cast<float>(wd[i]);
  float* d = nullptr;
  check_cuda(cudaMalloc(&d, sizeof(float) * w.size()), "cudaMalloc(W prefix)");
  check_cuda(cudaMemcpy(d, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice), "upload W prefix");
  ds.W_by_k[K] = d;
  return d;
}

int Engine::kernel_count_for(const KernelSet& ks, int max_kernels) const {
  const int k = select_kernel_count(ks.all_values.empty() ? ks.eigenvalues : ks.all_values, ks.trace, max_kernels,
                                    settings.kernel_energy_fraction);
  return std::min(k, ks.num_kernels());
}

double* Engine::ilt_cost_buffer(int n_masks) {
  if (n_masks > ilt_cost_cap) {
    cudaFree(ilt_cost_dev);
    ilt_cost_dev = nullptr;
    ilt_cost_cap = 0;
    check_cuda(cudaMalloc(&ilt_cost_dev, sizeof(double) * n_masks), "cudaMalloc(ilt costs)");
    ilt_cost_cap = n_masks;
  }
  return ilt_cost_dev;
}

void* Engine::workspace(size_t bytes) {
  if (ws_override) {
    if (bytes > ws_override_bytes) throw Error(HUV_ERR_OUT_OF_MEMORY, "plan workspace too small");
    return ws_override;
  }
  if (bytes > ws_bytes) {
    if (ws) cudaFree(ws);
    ws = nullptr;
    ws_bytes = 0;
    check_cuda(cudaMalloc(&ws, bytes), "cudaMalloc(workspace)");
    ws_bytes = bytes;
  }
  return ws;
}

int Engine::choose_eval_grid(const DeviceSet& ds, int requested, bool mixed) const {
  const int min_m = 4 * ds.hb + 1;
  const bool mixed_ok = [&](int m) {
    return (m == 160 || m == 192 || m == 384) && m <= n && huv_launch::xt_ok(m, ds.hb) &&
           huv_launch::xt_ok(m, 2 * ds.hb);
  }(requested);
  if (requested > 0) {
    if (((requested & (requested - 1)) != 0 && !(mixed && mixed_ok)) || requested > n || requested < min_m)
      throw Error(HUV_ERR_INVALID_PARAMETER, "eval_grid: must be a power of two (or 160 / 192 / 384 for the FFT "
                                             "and hybrid forms) with 4h < M <= N (h = " + std::to_string(ds.hb) + ")");
    return requested;
  }
  int m = 8;
  while (m < min_m) m <<= 1;
  m = std::min(m, n);
  if (mixed) {
    // a register-radix length between 4h and the next power of two
    for (int c : {160, 192, 384})
      if (c >= min_m && c < m && c < n && huv_launch::xt_ok(c, ds.hb) && huv_launch::xt_ok(c, 2 * ds.hb)) return c;
  }
  return m;
}

static size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

bool Engine::field_fused(const DeviceSet& ds, int M) const {
  const char* env = std::getenv("HUV_FIELD_PASS");
  return env && std::string(env) == "fused" && huv_launch::field_fused_ok(M, ds.hb);
}

void Engine::run_fft_form(const huv_batch& b, const DeviceSet& ds, int M, float* out, cudaStream_t st, int K_use,
                          const float* W_use) {
  const int lgn = ilog2(n), lgm = ilog2(M);  // lgm: rounded up where M is 160, 192 or 384
  const int B = ds.B, K = K_use > 0 ? K_use : ds.K, hb = ds.hb;
  const float* Wf = W_use ? W_use : ds.W;
  const bool coarse = M < n;
  const int h2 = 2 * hb, B2 = 2 * h2 + 1;
  const size_t in_elem = b.input_kind == HUV_INPUT_RASTER_U8
                             ? 1
                             : (b.input_kind == HUV_INPUT_RASTER_F32 ? 4 : (b.input_kind == HUV_INPUT_RECTS ? 0 : 8));
  // Per-clip workspace.
  const size_t per_x = align256(sizeof(float2) * n * B);
  const size_t per_m = align256(sizeof(float2) * B * B);
  const bool fused = field_fused(ds, M);
  const size_t per_t = align256(std::max(sizeof(float2) * static_cast<size_t>(K) * B * M,
                                         fused ? huv_launch::field_fused_part_bytes(M, K) : size_t(0)));
  const size_t per_i = coarse ? align256(sizeof(float) * M * M) : 0;
  const size_t per_x2 = coarse ? align256(sizeof(float2) * M * B2) : 0;
  const size_t per_c = coarse ? align256(sizeof(float2) * B2 * B2) : 0;
  const size_t per_t2 = coarse ? align256(sizeof(float2) * static_cast<size_t>(B2) * n) : 0;
  const size_t per_mean = align256(sizeof(float) * (1 + (B + 3) / 4));
  const size_t per_clip = per_x + per_m + per_t + per_i + per_x2 + per_c + per_t2 + per_mean;
  // a C2 step (256 clips) runs as one chunk of the engine's own workspace, so
  // the column pass (2 blocks per SM, 10 blocks per clip) fills whole waves
  const size_t budget = chunk_budget();
  const int chunk = balanced_chunk(static_cast<int>(std::max<size_t>(1, budget / per_clip)), b.n_clips);
  char* base = static_cast<char*>(workspace(per_clip * chunk + 4096));
  float2* X = reinterpret_cast<float2*>(base);
  float2* Mb = reinterpret_cast<float2*>(base + per_x * chunk);
  float2* T = reinterpret_cast<float2*>(base + (per_x + per_m) * chunk);
  float* IM = reinterpret_cast<float*>(base + (per_x + per_m + per_t) * chunk);
  float2* X2 = reinterpret_cast<float2*>(base + (per_x + per_m + per_t + per_i) * chunk);
  float2* C = reinterpret_cast<float2*>(base + (per_x + per_m + per_t + per_i + per_x2) * chunk);
  float2* T2 = reinterpret_cast<float2*>(base + (per_x + per_m + per_t + per_i + per_x2 + per_c) * chunk);
  float* mean = reinterpret_cast<float*>(base + (per_x + per_m + per_t + per_i + per_x2 + per_c + per_t2) * chunk);
  const float2* twn = twiddle_n(n);
  const float2* twm = twiddle_n(M);
  for (int c0 = 0; c0 < b.n_clips; c0 += chunk) {
    const int nc = std::min(chunk, b.n_clips - c0);
    const void* in = static_cast<const char*>(b.input) + in_elem * static_cast<size_t>(n) * n * c0;
    float* o = out + static_cast<size_t>(n) * n * c0;
    prof.begin("mask_band", st);
    if (b.input_kind == HUV_INPUT_RECTS)
      rect_band(c0, nc, hb, Wf, Mb, mean, st);
    else
      check_cuda(huv_launch::band_forward(in, b.input_kind, n, lgn, hb, nc, X, Mb,
                                          b.pixel_transfer ? ds.ptx : nullptr, Wf, mean, twn, st,
                                          row_digit_table(hb), dev_err),
                 "band_forward");
    prof.end(st);
    prof.launches += 2;
    if (fused) {
      // the partial sums of the kernel groups reuse T's bytes (K B M complex per clip)
      prof.begin("socs_field_fused", st);
      check_cuda(huv_launch::socs_field_fused(ds.kband, Mb, K, hb, M, nc, ds.keep, ds.flare, mean, coarse ? IM : o,
                                              nullptr, reinterpret_cast<float*>(T), twm, st),
                 "socs_field_fused");
      prof.end(st);
      prof.launches += huv_launch::field_fused_part_bytes(M, K) ? 2 : 1;
    } else {
      prof.begin("socs_rows_inv", st);
      check_cuda(huv_launch::socs_rows_x(ds.kband, 0.f, Mb, K, hb, M, nc, T, twm, st), "socs_rows");
      prof.end(st);
      prof.begin("socs_cols_inv", st);
      check_cuda(huv_launch::socs_cols_x(T, K, hb, M, nc, ds.keep, ds.flare, mean, coarse ? IM : o, 0, twm, st),
                 "socs_cols");
      prof.end(st);
      prof.launches += 2;
    }
    if (coarse) {
      prof.begin("interp_band", st);
      check_cuda(huv_launch::band_forward(IM, HUV_INPUT_RASTER_F32, M, lgm, h2, nc, X2, C, nullptr, nullptr,
                                          nullptr, twm, st, nullptr, nullptr),
                 "band_forward(interp)");
      prof.end(st);
      const float scale = 1.0f / (static_cast<float>(M) * static_cast<float>(M));
      prof.begin("interp_rows_cols", st);
      check_cuda(huv_launch::socs_rows_x(nullptr, scale, C, 1, h2, n, nc, T2, twn, st), "socs_rows(interp)");
      check_cuda(huv_launch::socs_cols_x(T2, 1, h2, n, nc, 1.f, 0.f, nullptr, o, 1, twn, st), "socs_cols(interp)");
      prof.end(st);
      prof.launches += 4;
    }
  }
}

void Engine::image_batch(const huv_batch& b, float* out, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(mu);
  if (b.n_clips < 0) throw Error(HUV_ERR_INVALID_PARAMETER, "n_clips: must be >= 0");
  if (b.n_clips == 0) return;
  if (!b.input || !out) throw Error(HUV_ERR_INVALID_PARAMETER, "input/out: null pointer");
  if (b.input_kind < 0 || b.input_kind > 3) throw Error(HUV_ERR_INVALID_PARAMETER, "input_kind: unknown");
  if (!std::isfinite(b.defocus_nm)) throw Error(HUV_ERR_INVALID_PARAMETER, "defocus_nm: must be finite");
  // device rasters are read with TMA and vector loads, images written with vector stores
  if ((reinterpret_cast<uintptr_t>(out) & 15u) != 0 ||
      (b.input_kind != HUV_INPUT_RECTS && (reinterpret_cast<uintptr_t>(b.input) & 15u) != 0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "input/out: device buffers must be 16-byte aligned");
  ensure_device();
  if (b.input_kind == HUV_INPUT_RECTS) upload_rects(b);
  DeviceSet& ds = device_set(b.defocus_nm == 0.0 ? 0.0 : b.defocus_nm);
  int form = b.form;
  // FFT and hybrid forms evaluate on the smallest supported grid above 4h
  // (160 or 192 where that beats the next power of two); the tcgen05
  // y-contraction tiles the grid by 128, so its automatic grid is a power of
  // two raised to 128 (still exact: any M > 4h is).
  const int Mp2 = choose_eval_grid(ds, form == HUV_FORM_TC || form == HUV_FORM_TC_ROWS ? b.eval_grid : 0);
  const int Mtc = (b.eval_grid == 0 && Mp2 < 128 && n >= 128) ? 128 : Mp2;
  const int M = (form == HUV_FORM_TC || form == HUV_FORM_TC_ROWS) ? Mp2 : choose_eval_grid(ds, b.eval_grid, true);
  if (form == HUV_FORM_AUTO) form = hybrid_supported(ds, M) ? HUV_FORM_HYBRID : HUV_FORM_FFT;
  if (form == HUV_FORM_HYBRID) {
    if (!hybrid_supported(ds, M)) throw Error(HUV_ERR_UNSUPPORTED, "hybrid form: band or grid outside what its kernels support");
    run_tc_form(b, ds, M, out, st, 0, nullptr, kTcCoreFftField);
  } else if (form == HUV_FORM_TC || form == HUV_FORM_TC_ROWS) {
    if (!tc_supported(ds, Mtc)) throw Error(HUV_ERR_UNSUPPORTED, "TC form: band or grid outside what its kernels support");
    run_tc_form(b, ds, Mtc, out, st, 0, nullptr, form == HUV_FORM_TC_ROWS ? kTcCoreGemmRows : kTcCoreFftRows);
  } else if (form == HUV_FORM_FFT) {
    run_fft_form(b, ds, M, out, st);
  } else {
    throw Error(HUV_ERR_INVALID_PARAMETER, "form: unknown");
  }
}

// Host buffers in, host buffers out.  The batch is cut into chunks that
// flow through a ring of three device slots: copy-in on one internal stream,
// the imaging on `st`, copy-out on another, ordered by events, so that the
// host->device copy of chunk i+1 and the device->host copy of chunk i-1
// overlap the imaging of chunk i (PCIe is full duplex).
void Engine::image_batch_host(const huv_batch& b, float* out_host, cudaStream_t st) {
  std::lock_guard<std::mutex> host_lock(host_mu);
  if (b.n_clips <= 0) return;
  if (!b.input || !out_host) throw Error(HUV_ERR_INVALID_PARAMETER, "input/out: null pointer");
  if (b.input_kind < 0 || b.input_kind > 3) throw Error(HUV_ERR_INVALID_PARAMETER, "input_kind: unknown");
  // Rectangle clips are read on the host (their tables are built there):
  // nothing to copy in, each chunk views its slice of the offsets.
  const bool rects = b.input_kind == HUV_INPUT_RECTS;
  const size_t in_elem = b.input_kind == HUV_INPUT_RASTER_U8
                             ? 1
                             : (b.input_kind == HUV_INPUT_RASTER_F32 ? 4 : (rects ? 0 : 8));
  const size_t in_per = in_elem * static_cast<size_t>(n) * n;
  const size_t out_per = sizeof(float) * static_cast<size_t>(n) * n;
  const int by_bytes = static_cast<int>(std::max<size_t>(1, (size_t(128) << 20) / out_per));
  const int chunk = std::max(1, std::min((b.n_clips + 3) / 4, by_bytes));
  // The first chunk is a quarter of the others, so that the copy-out stream
  // (the bound: images are 4x the bytes of u8 rasters) starts sooner.
  const int first = std::max(1, chunk / 4);
  std::vector<int> starts{0};
  while (starts.back() < b.n_clips) starts.push_back(std::min(b.n_clips, starts.back() + (starts.size() == 1 ? first : chunk)));
  const int nchunks = static_cast<int>(starts.size()) - 1;
  const int ring = std::min(nchunks, 3);
  {
    std::lock_guard<std::mutex> lock(mu);
    ensure_device();
    const size_t in_bytes = in_per * chunk * ring, out_bytes = out_per * chunk * ring;
    if (in_bytes > io_in_bytes) {
      if (io_in) cudaFree(io_in);
      io_in = nullptr;
      io_in_bytes = 0;
      check_cuda(cudaMalloc(&io_in, in_bytes), "cudaMalloc(io_in)");
      io_in_bytes = in_bytes;
    }
    if (out_bytes > io_out_bytes) {
      if (io_out) cudaFree(io_out);
      io_out = nullptr;
      io_out_bytes = 0;
      check_cuda(cudaMalloc(&io_out, out_bytes), "cudaMalloc(io_out)");
      io_out_bytes = out_bytes;
    }
    if (!io_h2d) {
      check_cuda(cudaStreamCreateWithFlags(&io_h2d, cudaStreamNonBlocking), "cudaStreamCreate(h2d)");
      check_cuda(cudaStreamCreateWithFlags(&io_d2h, cudaStreamNonBlocking), "cudaStreamCreate(d2h)");
      for (int r = 0; r < 3; ++r) {
        check_cuda(cudaEventCreateWithFlags(&io_ev[0][r], cudaEventDisableTiming), "cudaEventCreate");
        check_cuda(cudaEventCreateWithFlags(&io_ev[1][r], cudaEventDisableTiming), "cudaEventCreate");
        check_cuda(cudaEventCreateWithFlags(&io_ev[2][r], cudaEventDisableTiming), "cudaEventCreate");
      }
    }
  }
  cudaEvent_t* in_done = io_ev[0];
  cudaEvent_t* img_done = io_ev[1];
  cudaEvent_t* out_done = io_ev[2];
  for (int i = 0; i < nchunks; ++i) {
    const int slot = i % ring;
    const int c0 = starts[i], nc = starts[i + 1] - starts[i];
    char* din = static_cast<char*>(io_in) + in_per * chunk * slot;
    float* dout = reinterpret_cast<float*>(static_cast<char*>(io_out) + out_per * chunk * slot);
    // the input slot is free once the imaging of chunk i - ring has run
    if (i >= ring) check_cuda(cudaStreamWaitEvent(io_h2d, img_done[slot], 0), "wait(img)");
    if (!rects)
      check_cuda(cudaMemcpyAsync(din, static_cast<const char*>(b.input) + in_per * c0, in_per * nc,
                                 cudaMemcpyHostToDevice, io_h2d),
                 "H2D input");
    check_cuda(cudaEventRecord(in_done[slot], io_h2d), "record(in)");
    check_cuda(cudaStreamWaitEvent(st, in_done[slot], 0), "wait(in)");
    // the output slot is free once chunk i - ring has been copied out
    if (i >= ring) check_cuda(cudaStreamWaitEvent(st, out_done[slot], 0), "wait(out)");
    huv_batch d = b;
    d.n_clips = nc;
    d.input = din;
    huv_rect_clips view{};
    if (rects) {
      view = *static_cast<const huv_rect_clips*>(b.input);
      view.offsets += c0;
      d.input = &view;
    }
    image_batch(d, dout, st);
    check_cuda(cudaEventRecord(img_done[slot], st), "record(img)");
    check_cuda(cudaStreamWaitEvent(io_d2h, img_done[slot], 0), "wait(img)");
    check_cuda(cudaMemcpyAsync(out_host + static_cast<size_t>(n) * n * c0, dout, out_per * nc,
                               cudaMemcpyDeviceToHost, io_d2h),
               "D2H images");
    check_cuda(cudaEventRecord(out_done[slot], io_d2h), "record(out)");
  }
  check_cuda(cudaStreamSynchronize(io_d2h), "cudaStreamSynchronize(d2h)");
  check_cuda(cudaStreamSynchronize(io_h2d), "cudaStreamSynchronize(h2d)");
  check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  std::lock_guard<std::mutex> lock(mu);
  if (read_device_error() != 0)
    throw Error(HUV_ERR_DEVICE_TIMEOUT, "a bounded device-side wait gave up; the images are not valid");
}

int Engine::read_device_error() {
  if (!dev_err) return 0;
  int v = 0;
  check_cuda(cudaMemcpy(&v, dev_err, sizeof(int), cudaMemcpyDeviceToHost), "read device error flag");
  if (v) check_cuda(cudaMemset(dev_err, 0, sizeof(int)), "reset device error flag");
  return v;
}

}  // namespace huv
