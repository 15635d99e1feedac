// Engine state shared by the C ABI and the device launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "host/host.hpp"

namespace huv_launch {
// Band of the 2-D spectrum of `clips` rasters (csrc/cuda/socs_fft.cu): the
// one declaration every caller sees.
cudaError_t band_forward(const void* in, int kind, int n, int lg, int hb, int clips, float2* X, float2* Mband,
                         const float* ptx, const float* W, float* mean, const float2* tw, cudaStream_t st,
                         const uint8_t* row_digits, int* err);
}  // namespace huv_launch

namespace huv {

// Clips per chunk when a batch of n must be cut into chunks of at most
// max_chunk: the fewest chunks, sized evenly (216 + 40 becomes 128 + 128),
// so that the last chunk does not run the kernels on a partial wave.
inline int balanced_chunk(int max_chunk, int n) {
  if (n <= 0) return 1;
  max_chunk = max_chunk < 1 ? 1 : max_chunk;
  const int chunks = (n + max_chunk - 1) / max_chunk;
  return (n + chunks - 1) / chunks;
}

void set_last_error(const std::string& m);
const char* last_error();
void check_cuda(cudaError_t e, const char* what);

// Runs fn once per CUDA device for settings that CUDA keeps per device
// (function attributes): bit d of `done` is set after device d ran it.  Two
// threads may both run fn for one device; the calls it makes are idempotent.
template <class F>
void once_per_device(std::atomic<uint64_t>& done, F&& fn) {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  const uint64_t bit = dev >= 0 && dev < 64 ? (uint64_t(1) << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return;
  fn();
  if (bit) done.fetch_or(bit, std::memory_order_acq_rel);
}

// Device-side state of the tensor-core form for one kernel set: the split
// BF16 DFT operands (A_E over the evaluation grid, A_I for the interpolation
// to the output grid) and their TMA descriptors.
// How the tensor-core form evaluates sum lambda |E|^2 on the evaluation
// grid before its tcgen05 band interpolation: FP32 FFT row transforms into
// the split operand + the tcgen05 y-contraction (HUV_FORM_TC), both on
// tcgen05 (HUV_FORM_TC_ROWS), or the FP32 register-radix FFT field pass
// (HUV_FORM_HYBRID).
constexpr int kTcCoreFftRows = 0, kTcCoreGemmRows = 1, kTcCoreFftField = 2;

// Device state of the ILT optimizer (gradients, directions, trial masks,
// reductions), kept by the engine so that repeated optimizer calls do not
// allocate; every buffer only grows.
struct IltOptState {
  struct DevVec {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t b);
    template <typename T>
    T* as() const {
      return static_cast<T*>(p);
    }
  };
  DevVec grad, dir, gnew, trial, tgt, gold, cost_d, parts, dots, alpha, gamma, idx;
  void release();
};

struct TcState {
  int lgm = 0;          // evaluation grid the state was built for (log2, rounded up)
  void* gy = nullptr;   // A_E planes [2][2M][kpE] bf16
  void* gx = nullptr;   // A_I planes [2][N][kpI] bf16
  void* gp = nullptr;   // separable interpolation matrix planes [2][N][192] fp16 (M <= 192)
  CUtensorMap map_ae, map_ai, map_pi;
  CUtensorMap map_ai32, map_pi32;  // the same planes in 32-wide boxes (64B swizzle)
};

// One kernel set on the device: band kernels K x B x B (complex FP32,
// pre-scaled by sqrt(lambda_k / divisor) / N^2), the flare weight map W
// (B x B) and the pixel-transfer factors (B).
struct DeviceSet {
  const KernelSet* source = nullptr;
  // Keeps `source` alive while this copy refers to it, so a later set can
  // never be allocated at the same address and mistaken for it.
  std::shared_ptr<KernelSet> hold;
  int hb = 0, B = 0, K = 0;
  float keep = 1.f, flare = 0.f;
  float2* kband = nullptr;
  float* W = nullptr;
  float* ptx = nullptr;
  std::vector<double> eig_scaled;
  std::map<int, float*> W_by_k;  // flare weights of kernel-count prefixes
  std::vector<float2> host_kband;
  std::map<int, TcState> tc;  // per evaluation grid (log2 M); kept for the set's lifetime
};

// Launch accounting and live timing of the dominant kernel.  When `on`,
// each launch of the dominant kernel is bracketed by a pair of CUDA events
// recorded on the launching stream; `launches` counts every launch of this
// library's kernels.
struct Prof {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  std::vector<std::string> names;  // region name of each used event pair
  size_t used = 0;
  int64_t launches = 0;
  void begin(const char* nm, cudaStream_t st) {
    if (!on) return;
    if (used == pool.size()) {
      cudaEvent_t a, b;
      check_cuda(cudaEventCreate(&a), "cudaEventCreate");
      check_cuda(cudaEventCreate(&b), "cudaEventCreate");
      pool.emplace_back(a, b);
    }
    if (names.size() <= used) names.resize(used + 1);
    names[used] = nm;
    check_cuda(cudaEventRecord(pool[used].first, st), "cudaEventRecord");
  }
  void end(cudaStream_t st) {
    if (!on) return;
    check_cuda(cudaEventRecord(pool[used].second, st), "cudaEventRecord");
    ++used;
  }
  // name -> (launches, total ms) over the recorded regions
  std::map<std::string, std::pair<int, double>> regions() {
    std::map<std::string, std::pair<int, double>> out;
    for (size_t i = 0; i < used; ++i) {
      check_cuda(cudaEventSynchronize(pool[i].second), "cudaEventSynchronize");
      float ms = 0;
      check_cuda(cudaEventElapsedTime(&ms, pool[i].first, pool[i].second), "cudaEventElapsedTime");
      auto& r = out[names[i]];
      r.first += 1;
      r.second += ms;
    }
    return out;
  }
  void reset() {
    used = 0;
    launches = 0;
  }
  void release() {
    for (auto& pr : pool) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    pool.clear();
    names.clear();
    used = 0;
  }
};

// A learned image model usable inside ILT in place of the exact SOCS image.
struct Surrogate {
  virtual ~Surrogate() = default;
  virtual int grid() const = 0;
  // img[b] = model(t[b]) for B maps of grid x grid.
  virtual void forward(int B, const float* t, float* img, cudaStream_t st) = 0;
  // dt[b] = d sum(dout . model(t)) / dt.
  virtual void input_grad(int B, const float* t, const float* dout, float* dt, cudaStream_t st) = 0;
};

// Outcome of a surrogate-assisted ILT run.
struct SurrogateReport {
  int surrogate_iterations = 0;
  int exact_iterations = 0;
  int takeover_iteration = -1;       // iteration at which exact SOCS took over (-1: never)
  std::vector<double> judge_errors;  // max relative image error at each judge
};

struct CacheEntry {
  double z = 0;
  std::shared_ptr<KernelSet> ks;
  DeviceSet dev;
  uint64_t last_used = 0;
};

struct Engine {
  Engine(const huv_source& s, const huv_optics& o, const huv_grid& g, const huv_settings& st, int device);
  // An engine over a caller-supplied kernel set for one focus plane
  // (huv_kernelset_create): no source or optics, no other planes.
  Engine(const huv_kernel_set& set, int device);
  ~Engine();

  std::shared_ptr<KernelSet> kernel_set(double z);
  // The kernel set of plane z if the engine holds it already (the in-focus
  // set or a cached plane), else null; builds, evicts and allocates nothing.
  std::shared_ptr<KernelSet> held_set(double z);
  void cache_insert(double z, std::shared_ptr<KernelSet> ks);
  // The kernel set of focus plane z, built where settings.kernel_build says.
  KernelSet build_set(double z);
  void image_batch(const huv_batch& b, float* out, cudaStream_t st);
  void image_batch_host(const huv_batch& b, float* out_host, cudaStream_t st);
  // Rectangle clips (HUV_INPUT_RECTS): the batch's row/run table on the
  // device, then the exact band spectrum of clips [c0, c0 + nc).
  void upload_rects(const huv_batch& b);
  void rect_band(int c0, int nc, int hb, const float* W, float2* Mband, float* mean, cudaStream_t st);
  // Kernel sets of the focus planes not cached yet, built concurrently (one
  // plane per host thread) and cached.
  void prebuild_planes(const double* z, int planes);
  // out[plane][clip][y][x]: the batch imaged at every focus plane.
  void image_focus_sweep(const huv_batch& b, const double* z, int planes, float* out, cudaStream_t st);

  // device helpers
  void ensure_device();
  const float2* twiddle(int lg);
  // Twiddle table exp(-2 pi i t / L), t < L, for any supported length L.
  const float2* twiddle_n(int L);
  // Digit planes of the tensor-core row band of u8 rasters for band
  // half-width hb (NULL when that path does not apply to this grid, or when
  // HUV_MASK_ROWS=fft in the environment selects the FFT rows).
  const uint8_t* row_digit_table(int hb);
  DeviceSet& device_set(double z);
  void* workspace(size_t bytes);
  // Bytes a batch chunk may take of the workspace: 2 GiB of the engine's
  // own (a C2 step of 256 clips is one chunk), or what a captured plan's
  // workspace holds beyond the 4 KiB alignment slack every chunk adds.
  size_t chunk_budget() const {
    constexpr size_t kOwn = size_t(2) << 30, kSlack = 8192;
    if (!ws_override) return kOwn;
    return ws_override_bytes > kSlack ? ws_override_bytes - kSlack : 1;
  }
  // Device buffer of at least n doubles for per-mask ILT costs, kept (and
  // grown) for the engine's lifetime.
  double* ilt_cost_buffer(int n);
  double* ilt_cost_dev = nullptr;
  int ilt_cost_cap = 0;
  IltOptState ilt_state;
  // Evaluation grid M > 4h.  `mixed`: also the register-radix lengths 160
  // and 192 (the FFT and hybrid forms), else powers of two only.
  int choose_eval_grid(const DeviceSet& ds, int requested, bool mixed = false) const;
  // Whether the field pass on an M grid runs as the fused kernel (row and
  // column transforms of each kernel in one CTA, no HBM round trip) instead
  // of the row kernel + column kernel pair: only when HUV_FIELD_PASS=fused is
  // set in the environment (it measures slower than the pair), M = 128 or 160
  // and the band fits its shared memory.
  bool field_fused(const DeviceSet& ds, int M) const;
  // Whether the hybrid form (FFT field pass on M, tcgen05 interpolation) serves M.
  bool hybrid_supported(const DeviceSet& ds, int M) const;
  bool tc_supported(const DeviceSet& ds, int M) const;
  // K_use / W_use: kernel count and flare weights to use (0 / nullptr = the whole set).
  void run_fft_form(const huv_batch& b, const DeviceSet& ds, int M, float* out, cudaStream_t st, int K_use = 0,
                    const float* W_use = nullptr);
  void run_tc_form(const huv_batch& b, DeviceSet& ds, int M, float* out, cudaStream_t st, int K_use = 0,
                   const float* W_use = nullptr, int core = kTcCoreFftRows);
  // Separable band interpolation of nc coarse images to the N grid on
  // tcgen05: im_split holds I_M / interp_scale(mean) as FP16 hi/lo planes
  // [clip][2][M][M] (socs_cols_split), BI is 2 N M halves of workspace per
  // clip, out receives I_N = P I_M P^T.  Applies where separable_ok.
  bool separable_ok(const DeviceSet& ds, int M) const;
  void interp_matrix(DeviceSet& ds, int M);
  void interp_separable(DeviceSet& ds, int M, int nc, const void* im_split, const float* mean, void* BI, float* out,
                        cudaStream_t st, bool profile);
  // Flare weights W = sum_{k < K} lambda_k |u_k|^2 / N^4 of the first K kernels (device, cached).
  const float* flare_weights(DeviceSet& ds, int K);
  // Kernel count for a budget of `max_kernels` under the reference's truncation rule.
  int kernel_count_for(const KernelSet& ks, int max_kernels) const;
  // ILT (batched): cost and optional gradient; the optimizer.
  void ilt_eval(const huv_ilt_params& p, int masks, const float* theta, const float* target, float* grad,
                double* cost_dev, cudaStream_t st);
  void ilt_optimize(const huv_ilt_params& p, const huv_ilt_opt& o, int masks, float* theta, const float* target,
                    double* final_cost, int* iterations, double* history, cudaStream_t st,
                    Surrogate* sur = nullptr, int judge_every = 5, double error_bound = 0.05,
                    SurrogateReport* report = nullptr);
  // Cost (and gradient) with the image from `sur` instead of SOCS.
  void ilt_eval_surrogate(Surrogate* sur, const huv_ilt_params& p, int masks, const float* theta,
                          const float* target, float* grad, double* cost_dev, cudaStream_t st);
  // Max relative image error of the surrogate against SOCS, per mask (host).
  std::vector<double> surrogate_error(Surrogate* sur, const huv_ilt_params& p, int masks, const float* theta,
                                      cudaStream_t st);
  // Device error flag written by bounded waits that gave up (0 = none).
  int read_device_error();

  huv_settings settings;
  int device;
  // Engines over a caller-supplied set hold that one plane, at fixed_z.
  bool fixed_set = false;
  double fixed_z = 0.0;
  // The key a focus plane is held under: the fixed set's own plane is the
  // engine's plane 0; any other plane of a fixed set is refused.
  double plane_key(double z) const;
  Fill fill;
  Optics optics;
  int n = 0;
  double pixel_nm = 0, lambda = 0;
  std::vector<SourcePoint> points;
  std::shared_ptr<KernelSet> focus, scratch_set;
  std::vector<CacheEntry> cache;
  uint64_t clock = 0;

  Prof prof;
  std::mutex mu, host_mu;
  bool device_ready = false;
  std::map<int, float2*> twiddles;
  std::map<int, uint8_t*> row_digits;
  DeviceSet focus_dev, scratch_dev;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  // When set, workspace() hands out this buffer (a captured plan's own
  // workspace) and fails instead of reallocating.
  void* ws_override = nullptr;
  size_t ws_override_bytes = 0;
  int* dev_err = nullptr;
  void* io_in = nullptr;
  void* io_out = nullptr;
  size_t io_in_bytes = 0, io_out_bytes = 0;
  struct RectTable {
    void *clip_rows = nullptr, *rows = nullptr, *runs = nullptr, *coef = nullptr;
    size_t clip_rows_cap = 0, rows_cap = 0, runs_cap = 0, coef_cap = 0;
    int n_rows = 0;
    double2 dv{0, 0}, bg{0, 0};
  } rect;
  cudaStream_t io_h2d = nullptr, io_d2h = nullptr;
  cudaEvent_t io_ev[3][3] = {};  // [copy-in done, imaging done, copy-out done][ring slot]
};

}  // namespace huv
