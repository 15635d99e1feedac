// Allocation-free batched imaging: huv_image_batch_noalloc.
//
// Some callers cannot call cudaMalloc: an application that has handed the
// whole device to its own memory pool (serving stacks that reserve HBM up
// front), or a latency-critical loop that must not take cudaMalloc's implicit
// device-wide synchronisation.  For them this entry point runs the plain FP32
// FFT form with every intermediate buffer placed in one file-scope device
// array of fixed size (kNoAllocScratchBytes), and copies the kernel set into
// that same array on each call.  It never calls cudaMalloc, cudaFree or any
// allocating library routine.
//
// Set-up: the first call on a device takes the array's device address with
// cudaGetSymbolAddress (the host-side symbol is only a stand-in, not a device
// address) and sets the kernels' shared-memory limits.  Every GPU that loads
// the library holds the array until the process exits.
//
// All calls share the array, which keeps the last call's contents: calls
// that overlap on the GPU (different streams, or different host threads)
// race and must not be issued.  Each launch writes every scratch element it
// later reads, so nothing needs to start at zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "../../../include/huv_b200.h"
#include "../engine.hpp"

namespace huv_launch {
cudaError_t socs_rows(const float2* kband, float scale, const float2* Mband, int K, int hb, int lgm, int clips,
                      float2* T, const float2* tw, cudaStream_t st);
cudaError_t socs_cols(const float2* T, int K, int hb, int lgm, int clips, float keep, float flare,
                      const float* mean, float* out, int mode, const float2* tw, cudaStream_t st);
cudaError_t set_smem_limits();
}  // namespace huv_launch

namespace {

// Maximum scratch of the allocation-free entry point (32 MiB per device).
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: the array's device address.
void* scratch_for_device(int device) {
  if (device < 0 || device >= kMaxDevices)
    throw huv::Error(HUV_ERR_INVALID_PARAMETER, "device ordinal out of range for the allocation-free path");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    huv::check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
    huv::check_cuda(huv_launch::set_smem_limits(), "cudaFuncSetAttribute");
    g_scratch_ptr[device] = p;
  }
  return g_scratch_ptr[device];
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
int ilog2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

}  // namespace

extern "C" huv_status huv_image_batch_noalloc(void* engine, const huv_batch* batch, float* out, void* stream) {
  try {
    if (!engine || !batch) throw huv::Error(HUV_ERR_INVALID_PARAMETER, "engine/batch: null");
    huv::Engine* e = static_cast<huv::Engine*>(engine);
    const huv_batch& b = *batch;
    if (b.n_clips < 0) throw huv::Error(HUV_ERR_INVALID_PARAMETER, "n_clips: must be >= 0");
    if (b.n_clips == 0) {
      huv::set_last_error("");
      return HUV_OK;
    }
    if (!b.input || !out) throw huv::Error(HUV_ERR_INVALID_PARAMETER, "input/out: null pointer");
    if (b.input_kind < 0 || b.input_kind > 2) throw huv::Error(HUV_ERR_INVALID_PARAMETER, "input_kind: unknown");
    if ((reinterpret_cast<uintptr_t>(out) & 15u) != 0 || (reinterpret_cast<uintptr_t>(b.input) & 15u) != 0)
      throw huv::Error(HUV_ERR_INVALID_PARAMETER, "input/out: device buffers must be 16-byte aligned");
    if (b.form != HUV_FORM_AUTO && b.form != HUV_FORM_FFT)
      throw huv::Error(HUV_ERR_UNSUPPORTED, "the allocation-free path runs the FP32 FFT form only");
    if (!std::isfinite(b.defocus_nm)) throw huv::Error(HUV_ERR_INVALID_PARAMETER, "defocus_nm: must be finite");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(e->mu);
    huv::check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
    char* base = static_cast<char*>(scratch_for_device(e->device));

    // Host-side band kernels (pre-scaled like the engine's device set).  The
    // engine's plane cache is only read: a plane it does not hold is built
    // here on the host (FP64, as the engine's host build does) and dropped
    // after the call, never cached, so no device set is built or evicted.
    // An engine whose kernels are built on the GPU would need device memory
    // for that build, so it must hold the plane already.
    const double z = b.defocus_nm == 0.0 ? 0.0 : b.defocus_nm;
    std::shared_ptr<huv::KernelSet> ks = e->held_set(z);
    if (!ks) {
      if (e->settings.kernel_build != HUV_BUILD_HOST)
        throw huv::Error(HUV_ERR_UNSUPPORTED,
                         "allocation-free path: focus plane not cached, and this engine builds kernels on the GPU; "
                         "image the plane once with huv_image_batch (or huv_image_focus_sweep) first");
      ks = std::make_shared<huv::KernelSet>(huv::build_kernels(e->points, e->optics, e->n, e->pixel_nm, e->lambda,
                                                               e->settings.max_kernels,
                                                               e->settings.kernel_energy_fraction, z));
    }
    const int n = e->n;
    const int h = ks->band_half_width(), B = 2 * h + 1, K = ks->num_kernels();
    const int S = static_cast<int>(ks->support.size());
    double div = ks->divisor(e->settings.normalization);
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
        const huv::cd u = ks->values[static_cast<size_t>(k) * S + t];
        const size_t o = static_cast<size_t>(my + h) * B + (mx + h);
        kb[static_cast<size_t>(k) * B * B + o] =
            make_float2(static_cast<float>(u.real() * sc), static_cast<float>(u.imag() * sc));
        wd[o] += lam * std::norm(u) / (n2 * n2);
      }
    }
    std::vector<float> wf(wd.begin(), wd.end()), ptx(B);
    for (int i = 0; i < B; ++i) {
      const double u = 3.14159265358979323846 * (i - h) / n;
      ptx[i] = static_cast<float>(std::fabs(u) < 1e-6 ? 1.0 - u * u / 6.0 : std::sin(u) / u);
    }
    // Evaluation grid: as the engine chooses for the FFT form.
    int M = 8;
    while (M < 4 * h + 1) M <<= 1;
    M = std::min(M, n);
    if (b.eval_grid > 0) {
      if ((b.eval_grid & (b.eval_grid - 1)) != 0 || b.eval_grid > n || b.eval_grid < 4 * h + 1)
        throw huv::Error(HUV_ERR_INVALID_PARAMETER, "eval_grid: must be a power of two with 4h < M <= N");
      M = b.eval_grid;
    }
    const bool coarse = M < n;
    const int lgn = ilog2i(n), lgm = ilog2i(M);
    const int h2 = 2 * h, B2 = 2 * h2 + 1;
    auto twiddles = [](int L) {
      std::vector<float2> t(L);
      for (int i = 0; i < L; ++i) {
        const double a = -2.0 * 3.14159265358979323846 * i / L;
        t[i] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
      }
      return t;
    };
    const std::vector<float2> twn = twiddles(n), twm = twiddles(M);
    // Fixed part of the scratch: kernel set and twiddle tables.
    size_t off = 0;
    auto place = [&](size_t bytes) {
      char* p = base + off;
      off += align256(bytes);
      return p;
    };
    float2* d_kb = reinterpret_cast<float2*>(place(sizeof(float2) * kb.size()));
    float* d_w = reinterpret_cast<float*>(place(sizeof(float) * wf.size()));
    float* d_ptx = reinterpret_cast<float*>(place(sizeof(float) * ptx.size()));
    float2* d_twn = reinterpret_cast<float2*>(place(sizeof(float2) * twn.size()));
    float2* d_twm = reinterpret_cast<float2*>(place(sizeof(float2) * twm.size()));
    // Per-clip part.
    const size_t per_x = align256(sizeof(float2) * n * B);
    const size_t per_m = align256(sizeof(float2) * B * B);
    const size_t per_t = align256(sizeof(float2) * static_cast<size_t>(K) * B * M);
    const size_t per_i = coarse ? align256(sizeof(float) * M * M) : 0;
    const size_t per_x2 = coarse ? align256(sizeof(float2) * M * B2) : 0;
    const size_t per_c = coarse ? align256(sizeof(float2) * B2 * B2) : 0;
    const size_t per_t2 = coarse ? align256(sizeof(float2) * static_cast<size_t>(B2) * n) : 0;
    const size_t per_mean = align256(sizeof(float) * (1 + (B + 3) / 4));
    const size_t per_clip = per_x + per_m + per_t + per_i + per_x2 + per_c + per_t2 + per_mean;
    if (off + per_clip > kNoAllocScratchBytes)
      throw huv::Error(HUV_ERR_INVALID_PARAMETER,
                       "allocation-free path: one clip needs " + std::to_string((off + per_clip) >> 20) +
                           " MiB of scratch, above its fixed maximum of " +
                           std::to_string(kNoAllocScratchBytes >> 20) + " MiB; use huv_image_batch");
    const int chunk = huv::balanced_chunk(static_cast<int>((kNoAllocScratchBytes - off) / per_clip), b.n_clips);
    char* cb = base + off;
    float2* X = reinterpret_cast<float2*>(cb);
    float2* Mb = reinterpret_cast<float2*>(cb + per_x * chunk);
    float2* T = reinterpret_cast<float2*>(cb + (per_x + per_m) * chunk);
    float* IM = reinterpret_cast<float*>(cb + (per_x + per_m + per_t) * chunk);
    float2* X2 = reinterpret_cast<float2*>(cb + (per_x + per_m + per_t + per_i) * chunk);
    float2* C = reinterpret_cast<float2*>(cb + (per_x + per_m + per_t + per_i + per_x2) * chunk);
    float2* T2 = reinterpret_cast<float2*>(cb + (per_x + per_m + per_t + per_i + per_x2 + per_c) * chunk);
    float* mean = reinterpret_cast<float*>(cb + (per_x + per_m + per_t + per_i + per_x2 + per_c + per_t2) * chunk);
    huv::check_cuda(cudaMemcpyAsync(d_kb, kb.data(), sizeof(float2) * kb.size(), cudaMemcpyHostToDevice, st), "kband");
    huv::check_cuda(cudaMemcpyAsync(d_w, wf.data(), sizeof(float) * wf.size(), cudaMemcpyHostToDevice, st), "W");
    huv::check_cuda(cudaMemcpyAsync(d_ptx, ptx.data(), sizeof(float) * ptx.size(), cudaMemcpyHostToDevice, st), "ptx");
    huv::check_cuda(cudaMemcpyAsync(d_twn, twn.data(), sizeof(float2) * twn.size(), cudaMemcpyHostToDevice, st), "tw");
    huv::check_cuda(cudaMemcpyAsync(d_twm, twm.data(), sizeof(float2) * twm.size(), cudaMemcpyHostToDevice, st), "tw");
    const float flare = e->optics.flare > 0.0 ? static_cast<float>(e->optics.flare) : 0.f;
    const float keep = e->optics.flare > 0.0 ? static_cast<float>(1.0 - e->optics.flare) : 1.f;
    const size_t in_elem = b.input_kind == HUV_INPUT_RASTER_U8 ? 1 : (b.input_kind == HUV_INPUT_RASTER_F32 ? 4 : 8);
    for (int c0 = 0; c0 < b.n_clips; c0 += chunk) {
      const int nc = std::min(chunk, b.n_clips - c0);
      const void* in = static_cast<const char*>(b.input) + in_elem * static_cast<size_t>(n) * n * c0;
      float* o = out + static_cast<size_t>(n) * n * c0;
      huv::check_cuda(huv_launch::band_forward(in, b.input_kind, n, lgn, h, nc, X, Mb,
                                               b.pixel_transfer ? d_ptx : nullptr, d_w, mean, d_twn, st, nullptr,
                                               nullptr),
                      "band_forward");
      huv::check_cuda(huv_launch::socs_rows(d_kb, 0.f, Mb, K, h, lgm, nc, T, d_twm, st), "socs_rows");
      huv::check_cuda(huv_launch::socs_cols(T, K, h, lgm, nc, keep, flare, mean, coarse ? IM : o, 0, d_twm, st),
                      "socs_cols");
      if (coarse) {
        huv::check_cuda(huv_launch::band_forward(IM, HUV_INPUT_RASTER_F32, M, lgm, h2, nc, X2, C, nullptr, nullptr,
                                                 nullptr, d_twm, st, nullptr, nullptr),
                        "band_forward(interp)");
        const float scale = 1.0f / (static_cast<float>(M) * static_cast<float>(M));
        huv::check_cuda(huv_launch::socs_rows(nullptr, scale, C, 1, h2, lgn, nc, T2, d_twn, st), "socs_rows(interp)");
        huv::check_cuda(huv_launch::socs_cols(T2, 1, h2, lgn, nc, 1.f, 0.f, nullptr, o, 1, d_twn, st),
                        "socs_cols(interp)");
      }
    }
    huv::set_last_error("");
    return HUV_OK;
  } catch (const huv::Error& err) {
    huv::set_last_error(err.what());
    return err.status;
  } catch (const std::exception& err) {
    huv::set_last_error(err.what());
    return HUV_ERR_NUMERICAL;
  }
}
