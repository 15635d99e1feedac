// C ABI of the engine (include/huv_b200.h).  Every entry point catches
// exceptions, records the message for huv_last_error() and returns a status.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/huv_b200.h"
#include "engine.hpp"

using huv::Engine;
using huv::Error;

namespace {

template <typename F>
huv_status guarded(F&& f) {
  try {
    f();
    huv::set_last_error("");
    return HUV_OK;
  } catch (const Error& e) {
    huv::set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    huv::set_last_error("host allocation failed");
    return HUV_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    huv::set_last_error(e.what());
    return HUV_ERR_NUMERICAL;
  } catch (...) {
    huv::set_last_error("unknown failure");
    return HUV_ERR_NUMERICAL;
  }
}

void check_cuda_sync(Engine* e, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(e->mu);
  if (!e->device_ready) return;
  huv::check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
  huv::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (e->read_device_error() != 0)
    throw Error(HUV_ERR_DEVICE_TIMEOUT, "a bounded device-side wait gave up; results of the last calls are not valid");
}

void check_ilt_params(const huv_ilt_params& p) {
  auto pos = [](double v) { return std::isfinite(v) && v > 0; };
  if (p.cost_kind != 0 && p.cost_kind != 1) throw Error(HUV_ERR_INVALID_PARAMETER, "cost_kind: 0 or 1");
  if (!pos(p.beta)) throw Error(HUV_ERR_INVALID_PARAMETER, "sigmoid_steepness: must be positive and finite");
  if (!pos(p.tv_epsilon)) throw Error(HUV_ERR_INVALID_PARAMETER, "tv_epsilon: must be positive and finite");
  if (!(p.tv_weight >= 0) || !(p.binarization_weight >= 0))
    throw Error(HUV_ERR_INVALID_PARAMETER, "regularization weights: must be non-negative");
  if (p.cost_kind == 1 && (!pos(p.threshold) || !pos(p.steepness)))
    throw Error(HUV_ERR_INVALID_PARAMETER, "threshold/steepness: must be positive and finite");
  if (!pos(p.dose) || !(p.weight >= 0) || !std::isfinite(p.defocus_nm))
    throw Error(HUV_ERR_INVALID_PARAMETER, "condition: dose > 0, weight >= 0, finite defocus");
  if (!(p.absorber >= 0 && p.absorber < 1)) throw Error(HUV_ERR_INVALID_PARAMETER, "absorber: real, in [0, 1)");
}

Engine* as_engine(void* e) {
  if (!e) throw Error(HUV_ERR_INVALID_PARAMETER, "engine: null handle");
  return static_cast<Engine*>(e);
}

}  // namespace

extern "C" {

const char* huv_last_error(void) { return huv::last_error(); }
const char* huv_version(void) { return "highuvlith_b200 0.1.0 (sm_100a)"; }

huv_status huv_engine_create(const huv_source* source, const huv_optics* optics, const huv_grid* grid,
                             const huv_settings* settings, int32_t device, void** engine_out) {
  return guarded([&] {
    if (!source || !optics || !grid || !settings || !engine_out)
      throw Error(HUV_ERR_INVALID_PARAMETER, "huv_engine_create: null argument");
    *engine_out = nullptr;
    *engine_out = new Engine(*source, *optics, *grid, *settings, device);
  });
}

huv_status huv_kernelset_create(const huv_kernel_set* set, int32_t device, void** engine_out) {
  return guarded([&] {
    if (!set || !engine_out) throw Error(HUV_ERR_INVALID_PARAMETER, "huv_kernelset_create: null argument");
    *engine_out = nullptr;
    *engine_out = new Engine(*set, device);
  });
}

void huv_engine_destroy(void* engine) { delete static_cast<Engine*>(engine); }

huv_status huv_engine_source_points(void* engine, double* xyw, int32_t capacity, int32_t* count) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!count) throw Error(HUV_ERR_INVALID_PARAMETER, "count: null");
    *count = static_cast<int32_t>(e->points.size());
    if (!xyw) return;
    if (capacity < *count) throw Error(HUV_ERR_DIMENSION_MISMATCH, "source_points: capacity too small");
    for (size_t i = 0; i < e->points.size(); ++i) {
      xyw[3 * i] = e->points[i].sx;
      xyw[3 * i + 1] = e->points[i].sy;
      xyw[3 * i + 2] = e->points[i].w;
    }
  });
}

huv_status huv_engine_diagnostics(void* engine, double defocus_nm, huv_diagnostics* out) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!out) throw Error(HUV_ERR_INVALID_PARAMETER, "out: null");
    std::lock_guard<std::mutex> lock(e->mu);
    auto ks = e->kernel_set(defocus_nm);
    out->num_kernels = ks->num_kernels();
    out->captured_energy_fraction = [&] {
      double s = 0;
      for (double v : ks->eigenvalues) s += v;
      return s / ks->trace;
    }();
    out->num_frequencies = static_cast<int32_t>(ks->support.size());
    out->num_columns = ks->num_columns;
    out->method = ks->method;
    out->support_exceeds_nyquist = ks->exceeds_nyquist ? 1 : 0;
    out->clear_field_intensity = ks->clear_field;
    out->normalized = ks->divisor(e->settings.normalization) != 0.0 ? 1 : 0;
    out->band_half_width = ks->band_half_width();
    out->num_source_points = static_cast<int32_t>(e->points.size());
  });
}

huv_status huv_engine_clear_field(void* engine, double defocus_nm, double* out) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!out) throw Error(HUV_ERR_INVALID_PARAMETER, "out: null");
    std::lock_guard<std::mutex> lock(e->mu);
    *out = e->kernel_set(defocus_nm)->clear_field;
  });
}

huv_status huv_engine_kernels(void* engine, double defocus_nm, double* eigenvalues, double* kernels,
                              int32_t capacity, int32_t* count) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!count) throw Error(HUV_ERR_INVALID_PARAMETER, "count: null");
    std::lock_guard<std::mutex> lock(e->mu);
    auto ks = e->kernel_set(defocus_nm);
    const int K = ks->num_kernels();
    *count = K;
    if (!eigenvalues && !kernels) return;
    if (capacity < K) throw Error(HUV_ERR_DIMENSION_MISMATCH, "kernels: capacity too small");
    double div = ks->divisor(e->settings.normalization);
    if (div == 0.0) div = 1.0;
    const size_t nn = static_cast<size_t>(e->n) * e->n;
    const size_t S = ks->support.size();
    if (eigenvalues)
      for (int k = 0; k < K; ++k) eigenvalues[k] = ks->eigenvalues[k] / div;
    if (kernels) {
      std::memset(kernels, 0, sizeof(double) * 2 * nn * K);
      for (int k = 0; k < K; ++k)
        for (size_t t = 0; t < S; ++t) {
          const auto v = ks->values[k * S + t];
          const size_t o = (static_cast<size_t>(k) * nn + static_cast<size_t>(ks->support[t])) * 2;
          kernels[o] = v.real();
          kernels[o + 1] = v.imag();
        }
    }
  });
}

huv_status huv_image_batch(void* engine, const huv_batch* batch, float* out, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!batch) throw Error(HUV_ERR_INVALID_PARAMETER, "batch: null");
    e->image_batch(*batch, out, static_cast<cudaStream_t>(stream));
  });
}

huv_status huv_image_batch_host(void* engine, const huv_batch* batch, float* out_host, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!batch) throw Error(HUV_ERR_INVALID_PARAMETER, "batch: null");
    e->image_batch_host(*batch, out_host, static_cast<cudaStream_t>(stream));
  });
}

huv_status huv_image_focus_sweep(void* engine, const huv_batch* batch, const double* focus_nm, int32_t n_planes,
                                 float* out, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!batch) throw Error(HUV_ERR_INVALID_PARAMETER, "batch: null");
    e->image_focus_sweep(*batch, focus_nm, n_planes, out, static_cast<cudaStream_t>(stream));
  });
}

huv_status huv_ilt_cost_grad(void* engine, const huv_ilt_params* params, int32_t n_masks, const float* theta,
                             const float* target, double* cost_host, float* grad, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!params || !theta || !target || !cost_host) throw Error(HUV_ERR_INVALID_PARAMETER, "ilt: null argument");
    check_ilt_params(*params);
    if (n_masks <= 0) return;
    std::lock_guard<std::mutex> lock(e->mu);
    e->ensure_device();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* d = e->ilt_cost_buffer(n_masks);
    e->ilt_eval(*params, n_masks, theta, target, grad, d, st);
    huv::check_cuda(cudaMemcpyAsync(cost_host, d, sizeof(double) * n_masks, cudaMemcpyDeviceToHost, st), "D2H cost");
    huv::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  });
}

huv_status huv_ilt_optimize(void* engine, const huv_ilt_params* params, const huv_ilt_opt* opt, int32_t n_masks,
                            float* theta, const float* target, double* final_cost, int32_t* iterations,
                            double* history, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!params || !opt || !theta || !target) throw Error(HUV_ERR_INVALID_PARAMETER, "ilt: null argument");
    check_ilt_params(*params);
    if (opt->max_iterations < 0 || !(opt->learning_rate > 0) || !(opt->convergence_tol >= 0))
      throw Error(HUV_ERR_INVALID_PARAMETER, "ilt optimizer: max_iterations >= 0, learning_rate > 0, tol >= 0");
    if (n_masks <= 0) return;
    std::lock_guard<std::mutex> lock(e->mu);
    e->ensure_device();
    e->ilt_optimize(*params, *opt, n_masks, theta, target, final_cost, iterations, history,
                    static_cast<cudaStream_t>(stream));
  });
}

huv_status huv_device_status(void* engine, void* stream) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    check_cuda_sync(e, static_cast<cudaStream_t>(stream));
  });
}

huv_status huv_profile_enable(void* engine, int32_t on) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    std::lock_guard<std::mutex> lock(e->mu);
    e->prof.on = on != 0;
    e->prof.reset();
  });
}

huv_status huv_profile_read(void* engine, double* dominant_ms, int32_t* dominant_launches, int64_t* total_launches,
                            char* dominant_name, int32_t name_capacity) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    std::lock_guard<std::mutex> lock(e->mu);
    const auto regions = e->prof.regions();
    std::string best;
    double best_ms = 0.0;
    int best_n = 0;
    for (const auto& kv : regions)
      if (kv.second.second > best_ms) {
        best = kv.first;
        best_ms = kv.second.second;
        best_n = kv.second.first;
      }
    if (dominant_ms) *dominant_ms = best_ms;
    if (dominant_launches) *dominant_launches = best_n;
    if (total_launches) *total_launches = e->prof.launches;
    if (dominant_name && name_capacity > 0) {
      std::strncpy(dominant_name, best.c_str(), static_cast<size_t>(name_capacity) - 1);
      dominant_name[name_capacity - 1] = 0;
    }
    e->prof.reset();
  });
}

huv_status huv_profile_regions(void* engine, char* json, int32_t capacity) {
  return guarded([&] {
    Engine* e = as_engine(engine);
    if (!json || capacity <= 0) throw Error(HUV_ERR_INVALID_PARAMETER, "profile regions: buffer");
    std::lock_guard<std::mutex> lock(e->mu);
    std::string out = "{";
    bool first = true;
    for (const auto& kv : e->prof.regions()) {
      out += (first ? "\"" : ",\"") + kv.first + "\":[" + std::to_string(kv.second.first) + "," +
             std::to_string(kv.second.second) + "]";
      first = false;
    }
    out += "}";
    if (static_cast<int32_t>(out.size()) >= capacity) throw Error(HUV_ERR_DIMENSION_MISMATCH, "profile regions: capacity");
    std::memcpy(json, out.c_str(), out.size() + 1);
  });
}

}  // extern "C"
