// Uneven batches in one CUDA-graph launch, with an autotuner.
//
// A plan takes clips of different grids, sources and kernel budgets (each
// clip names the engine built for its source and grid, and its own
// max_kernels, re-truncated with the reference's cluster rule), groups them
// by (engine, kernel count, input kind), picks per group the device form and
// evaluation grid (tensor-core or FFT, coarse or full grid) by timing the
// candidates on the group's own clips, pre-allocates every buffer, runs the
// whole batch once, and captures it into a CUDA graph.  huv_plan_launch is
// then one cudaGraphLaunch for the whole uneven batch.  Tuning results are
// cached per (grid, band, kernel count, input kind) for the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/huv_b200.h"
#include "engine.hpp"

namespace huv_launch {
cudaError_t plan_copy(const void* const* src, void* const* dst, size_t bytes, int count, cudaStream_t st);
}

namespace huv {

namespace {

struct Choice {
  int form = HUV_FORM_FFT;
  int M = 0;
  double ms_per_clip = 0;
};

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, Choice> g_tuned;  // (N, h, K, kind) -> choice

size_t elem_size(int kind) { return kind == HUV_INPUT_RASTER_U8 ? 1 : (kind == HUV_INPUT_RASTER_F32 ? 4 : 8); }

struct Group {
  Engine* e = nullptr;
  int K = 0, kind = 0, n = 0, h = 0;
  std::vector<int> clips;
  Choice choice;
  const float* W = nullptr;
  bool contiguous = false;
  const void* in_base = nullptr;
  float* out_base = nullptr;
  void* stage_in = nullptr;
  float* stage_out = nullptr;
  // device pointer arrays of the gather / scatter kernel (non-contiguous
  // groups whose buffers and clip sizes are 16-byte aligned)
  bool copy_kernel = false;
  const void** gather_src = nullptr;
  void** gather_dst = nullptr;
  const void** scatter_src = nullptr;
  void** scatter_dst = nullptr;
};

}  // namespace

struct Plan {
  int device = 0;
  int pixel_transfer = 1;
  std::vector<huv_clip> clips;
  std::vector<Group> groups;
  // Branches of the captured graph: groups are spread over up to kBranches
  // streams (largest estimated work first, each to the least loaded
  // branch), each branch with its own workspace, so that groups too small
  // to fill the GPU run beside each other.
  static constexpr int kBranches = 4;
  std::vector<void*> ws;
  size_t ws_bytes = 0;
  std::vector<int> branch;  // per group
  std::vector<cudaStream_t> bstream;
  std::vector<cudaEvent_t> bevent;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string report;

  ~Plan() {
    cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& g : groups) {
      cudaFree(g.stage_in);
      cudaFree(g.stage_out);
      cudaFree(const_cast<void**>(g.gather_src));  // one allocation holds all four arrays
    }
    for (void* w : ws) cudaFree(w);
    for (cudaStream_t b : bstream) cudaStreamDestroy(b);
    for (cudaEvent_t e : bevent) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }

  // Run one group (inputs staged contiguously unless already so).
  void run_group(Group& g, const Choice& c, cudaStream_t st, int limit = -1) {
    const size_t in_bytes = elem_size(g.kind) * static_cast<size_t>(g.n) * g.n;
    const size_t out_bytes = sizeof(float) * static_cast<size_t>(g.n) * g.n;
    const int count = limit > 0 ? std::min<int>(limit, static_cast<int>(g.clips.size()))
                                : static_cast<int>(g.clips.size());
    const void* in = g.contiguous ? g.in_base : g.stage_in;
    float* out = g.contiguous ? g.out_base : g.stage_out;
    if (!g.contiguous) {
      if (g.copy_kernel)
        check_cuda(huv_launch::plan_copy(g.gather_src, g.gather_dst, in_bytes, count, st), "plan gather");
      else
        for (int i = 0; i < count; ++i)
          check_cuda(cudaMemcpyAsync(static_cast<char*>(g.stage_in) + in_bytes * i, clips[g.clips[i]].input,
                                     in_bytes, cudaMemcpyDeviceToDevice, st),
                     "plan gather");
    }
    huv_batch b{};
    b.n_clips = count;
    b.input_kind = g.kind;
    b.input = in;
    b.pixel_transfer = pixel_transfer;
    b.defocus_nm = 0.0;
    b.form = c.form;
    b.eval_grid = c.M;
    DeviceSet& ds = g.e->device_set(0.0);
    if (c.form == HUV_FORM_TC)
      g.e->run_tc_form(b, ds, c.M, out, st, g.K, g.W);
    else if (c.form == HUV_FORM_HYBRID)
      g.e->run_tc_form(b, ds, c.M, out, st, g.K, g.W, kTcCoreFftField);
    else
      g.e->run_fft_form(b, ds, c.M, out, st, g.K, g.W);
    if (!g.contiguous) {
      if (g.copy_kernel)
        check_cuda(huv_launch::plan_copy(g.scatter_src, g.scatter_dst, out_bytes, count, st), "plan scatter");
      else
        for (int i = 0; i < count; ++i)
          check_cuda(cudaMemcpyAsync(clips[g.clips[i]].out, reinterpret_cast<char*>(g.stage_out) + out_bytes * i,
                                     out_bytes, cudaMemcpyDeviceToDevice, st),
                     "plan scatter");
    }
  }
};

namespace {

std::vector<Choice> candidates(Engine* e, DeviceSet& ds) {
  std::vector<Choice> out;
  const int n = e->n;
  int m = 8;
  while (m < 4 * ds.hb + 1) m <<= 1;
  m = std::min(m, n);
  const int mtc = std::max(m, 128);
  // the FFT and hybrid forms may evaluate on a register-radix grid (160, 192, 384)
  // between 4h and the next power of two
  const int mx = e->choose_eval_grid(ds, 0, true);
  if (mtc <= n && e->tc_supported(ds, mtc)) out.push_back(Choice{HUV_FORM_TC, mtc, 0});
  if (e->hybrid_supported(ds, mx)) out.push_back(Choice{HUV_FORM_HYBRID, mx, 0});
  if (mx != m) out.push_back(Choice{HUV_FORM_FFT, mx, 0});
  out.push_back(Choice{HUV_FORM_FFT, m, 0});
  if (2 * m <= n && m < n) out.push_back(Choice{HUV_FORM_FFT, 2 * m, 0});
  if (m < n && out.size() < 5) out.push_back(Choice{HUV_FORM_FFT, n, 0});
  return out;
}

}  // namespace

}  // namespace huv

using huv::Engine;
using huv::Error;
using huv::Plan;

extern "C" {

huv_status huv_plan_create(const huv_clip* clips, int32_t n_clips, int32_t pixel_transfer, int32_t autotune,
                           void** plan_out) {
  Plan* plan = nullptr;
  try {
    if (!clips || n_clips <= 0 || !plan_out) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: clips/n_clips/plan_out");
    *plan_out = nullptr;
    plan = new Plan();
    plan->pixel_transfer = pixel_transfer ? 1 : 0;
    plan->clips.assign(clips, clips + n_clips);
    Engine* e0 = static_cast<Engine*>(clips[0].engine);
    if (!e0) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: null engine");
    plan->device = e0->device;
    huv::check_cuda(cudaSetDevice(plan->device), "cudaSetDevice");
    // group
    std::map<std::tuple<Engine*, int, int>, int> key_to_group;
    for (int i = 0; i < n_clips; ++i) {
      const huv_clip& c = clips[i];
      Engine* e = static_cast<Engine*>(c.engine);
      if (!e || !c.input || !c.out) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: null engine/input/out in a clip");
      if (e->device != plan->device) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: engines on different devices");
      if (c.input_kind < 0 || c.input_kind > 2) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: input_kind");
      if (c.max_kernels < 1) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: max_kernels must be >= 1");
      int K;
      {
        std::lock_guard<std::mutex> lock(e->mu);
        K = e->kernel_count_for(*e->kernel_set(0.0), c.max_kernels);
      }
      auto key = std::make_tuple(e, K, static_cast<int>(c.input_kind));
      auto it = key_to_group.find(key);
      if (it == key_to_group.end()) {
        huv::Group g;
        g.e = e;
        g.K = K;
        g.kind = c.input_kind;
        g.n = e->n;
        it = key_to_group.emplace(key, static_cast<int>(plan->groups.size())).first;
        plan->groups.push_back(g);
      }
      plan->groups[it->second].clips.push_back(i);
    }
    // per group: device state, contiguity, autotuning
    std::ostringstream rep;
    rep << "[";
    huv::check_cuda(cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaStream_t st = plan->stream;
    for (size_t gi = 0; gi < plan->groups.size(); ++gi) {
      huv::Group& g = plan->groups[gi];
      std::lock_guard<std::mutex> lock(g.e->mu);
      g.e->ensure_device();
      huv::DeviceSet& ds = g.e->device_set(0.0);
      g.h = ds.hb;
      g.W = g.e->flare_weights(ds, g.K);
      const size_t in_bytes = huv::elem_size(g.kind) * static_cast<size_t>(g.n) * g.n;
      const size_t out_bytes = sizeof(float) * static_cast<size_t>(g.n) * g.n;
      g.contiguous = true;
      for (size_t j = 1; j < g.clips.size() && g.contiguous; ++j) {
        const huv_clip& a = clips[g.clips[j - 1]];
        const huv_clip& b = clips[g.clips[j]];
        g.contiguous = static_cast<const char*>(b.input) == static_cast<const char*>(a.input) + in_bytes &&
                       reinterpret_cast<char*>(b.out) == reinterpret_cast<char*>(a.out) + out_bytes;
      }
      g.in_base = clips[g.clips[0]].input;
      g.out_base = clips[g.clips[0]].out;
      if (!g.contiguous) {
        huv::check_cuda(cudaMalloc(&g.stage_in, in_bytes * g.clips.size()), "cudaMalloc(plan stage in)");
        huv::check_cuda(cudaMalloc(reinterpret_cast<void**>(&g.stage_out), out_bytes * g.clips.size()),
                        "cudaMalloc(plan stage out)");
        const size_t nc = g.clips.size();
        bool aligned = in_bytes % 16 == 0 && out_bytes % 16 == 0 && nc <= 65535;
        for (size_t j = 0; j < nc && aligned; ++j)
          aligned = (reinterpret_cast<uintptr_t>(clips[g.clips[j]].input) & 15u) == 0 &&
                    (reinterpret_cast<uintptr_t>(clips[g.clips[j]].out) & 15u) == 0;
        if (aligned) {
          std::vector<const void*> ptrs(4 * nc);
          for (size_t j = 0; j < nc; ++j) {
            ptrs[j] = clips[g.clips[j]].input;                                              // gather src
            ptrs[nc + j] = static_cast<const char*>(g.stage_in) + in_bytes * j;             // gather dst
            ptrs[2 * nc + j] = reinterpret_cast<const char*>(g.stage_out) + out_bytes * j;  // scatter src
            ptrs[3 * nc + j] = clips[g.clips[j]].out;                                       // scatter dst
          }
          void** d = nullptr;
          huv::check_cuda(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(void*) * 4 * nc),
                          "cudaMalloc(plan copy pointers)");
          huv::check_cuda(cudaMemcpy(d, ptrs.data(), sizeof(void*) * 4 * nc, cudaMemcpyHostToDevice),
                          "upload plan copy pointers");
          g.gather_src = const_cast<const void**>(d);
          g.gather_dst = d + nc;
          g.scatter_src = const_cast<const void**>(d + 2 * nc);
          g.scatter_dst = d + 3 * nc;
          g.copy_kernel = true;
        }
      }
      const auto key = std::make_tuple(g.n, g.h, g.K, g.kind);
      bool cached = false;
      {
        std::lock_guard<std::mutex> tl(huv::g_tune_mu);
        auto it = huv::g_tuned.find(key);
        if (it != huv::g_tuned.end()) {
          g.choice = it->second;
          cached = true;
        }
      }
      const std::vector<huv::Choice> cands = huv::candidates(g.e, ds);
      if (!cached) {
        if (!autotune) {
          g.choice = cands.front();
        } else {
          // a sample large enough to fill the GPU (at least 32 clips or
          // 256 MB of images): with a handful of clips the launches' fixed
          // cost dominates and favours the forms with the fewest launches
          // (e.g. the full grid over a coarse grid plus interpolation), which
          // lose at the group's real size
          const size_t img_bytes = sizeof(float) * static_cast<size_t>(g.n) * g.n;
          const int want = static_cast<int>(std::max<size_t>(32, (size_t(256) << 20) / img_bytes));
          const int probe = std::min<int>(want, static_cast<int>(g.clips.size()));
          cudaEvent_t e0, e1;
          huv::check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
          huv::check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
          double best = 1e300;
          for (const huv::Choice& c : cands) {
            plan->run_group(g, c, st, probe);  // warm-up (sizes workspaces, builds operands)
            huv::check_cuda(cudaEventRecord(e0, st), "cudaEventRecord");
            for (int r = 0; r < 2; ++r) plan->run_group(g, c, st, probe);
            huv::check_cuda(cudaEventRecord(e1, st), "cudaEventRecord");
            huv::check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0;
            huv::check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            const double per = ms / (2.0 * probe);
            if (per < best) {
              best = per;
              g.choice = c;
              g.choice.ms_per_clip = per;
            }
          }
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
        }
        std::lock_guard<std::mutex> tl(huv::g_tune_mu);
        huv::g_tuned[key] = g.choice;
      }
      rep << (gi ? "," : "") << "{\"n\":" << g.n << ",\"h\":" << g.h << ",\"K\":" << g.K << ",\"clips\":"
          << g.clips.size() << ",\"form\":\"" << (g.choice.form == HUV_FORM_TC ? "tc" : (g.choice.form == HUV_FORM_HYBRID ? "hybrid" : "fft")) << "\",\"eval_grid\":"
          << g.choice.M << ",\"ms_per_clip\":" << g.choice.ms_per_clip << ",\"contiguous\":" << (g.contiguous ? 1 : 0)
          << "}";
    }
    rep << "]";
    plan->report = rep.str();
    // Branch assignment: estimated work = clips x the tuned ms per clip
    // (clips alone when not tuned), largest first, each to the branch with
    // the least work so far.
    const int nb = std::min<int>(Plan::kBranches, static_cast<int>(plan->groups.size()));
    {
      std::vector<int> order(plan->groups.size());
      for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
      auto work = [&](int i) {
        const auto& g = plan->groups[i];
        return static_cast<double>(g.clips.size()) * (g.choice.ms_per_clip > 0 ? g.choice.ms_per_clip : 1.0);
      };
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
      std::vector<double> load(nb, 0.0);
      plan->branch.assign(plan->groups.size(), 0);
      for (int i : order) {
        const int b = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        plan->branch[i] = b;
        load[b] += work(i);
      }
    }
    // One workspace per branch (groups of a branch run one after another):
    // as large as an engine's own chunk budget plus the per-chunk slack, so
    // each group's chunks are those of its standalone runs (every chunking
    // in the engine sizes itself by Engine::chunk_budget()).
    const size_t wsb = (size_t(2) << 30) + 8192;
    plan->ws.assign(nb, nullptr);
    for (int b = 0; b < nb; ++b) huv::check_cuda(cudaMalloc(&plan->ws[b], wsb), "cudaMalloc(plan workspace)");
    plan->ws_bytes = wsb;
    plan->bstream.assign(nb, nullptr);
    plan->bevent.assign(nb + 1, nullptr);
    for (int b = 0; b < nb; ++b)
      huv::check_cuda(cudaStreamCreateWithFlags(&plan->bstream[b], cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : plan->bevent)
      huv::check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    auto clear_ws = [&] {
      for (auto& g : plan->groups) g.e->ws_override = nullptr;
    };
    auto run_on = [&](huv::Group& g, int b, cudaStream_t s) {
      std::lock_guard<std::mutex> lock(g.e->mu);
      g.e->ws_override = plan->ws[b];
      g.e->ws_override_bytes = plan->ws_bytes;
      plan->run_group(g, g.choice, s);
    };
    try {
      // Full run, branch by branch on one stream (allocates every lazy operand).
      for (size_t gi = 0; gi < plan->groups.size(); ++gi) run_on(plan->groups[gi], plan->branch[gi], st);
      huv::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize(plan)");
      // Capture: fork the branches off `st`, run each branch's groups on
      // its stream, join them back.
      huv::check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      try {
        huv::check_cuda(cudaEventRecord(plan->bevent[nb], st), "cudaEventRecord(fork)");
        for (int b = 0; b < nb; ++b)
          huv::check_cuda(cudaStreamWaitEvent(plan->bstream[b], plan->bevent[nb], 0), "cudaStreamWaitEvent(fork)");
        for (size_t gi = 0; gi < plan->groups.size(); ++gi) {
          const int b = plan->branch[gi];
          run_on(plan->groups[gi], b, plan->bstream[b]);
        }
        for (int b = 0; b < nb; ++b) {
          huv::check_cuda(cudaEventRecord(plan->bevent[b], plan->bstream[b]), "cudaEventRecord(join)");
          huv::check_cuda(cudaStreamWaitEvent(st, plan->bevent[b], 0), "cudaStreamWaitEvent(join)");
        }
      } catch (...) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(st, &dead);
        if (dead) cudaGraphDestroy(dead);
        throw;
      }
      huv::check_cuda(cudaStreamEndCapture(st, &plan->graph), "cudaStreamEndCapture");
      huv::check_cuda(cudaGraphInstantiate(&plan->exec, plan->graph, 0), "cudaGraphInstantiate");
    } catch (...) {
      clear_ws();
      throw;
    }
    clear_ws();
    *plan_out = plan;
    huv::set_last_error("");
    return HUV_OK;
  } catch (const Error& e) {
    delete plan;
    huv::set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    delete plan;
    huv::set_last_error(e.what());
    return HUV_ERR_NUMERICAL;
  }
}

huv_status huv_plan_launch(void* plan, void* stream) {
  try {
    if (!plan) throw Error(HUV_ERR_INVALID_PARAMETER, "plan: null");
    Plan* p = static_cast<Plan*>(plan);
    huv::check_cuda(cudaSetDevice(p->device), "cudaSetDevice");
    huv::check_cuda(cudaGraphLaunch(p->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch");
    huv::set_last_error("");
    return HUV_OK;
  } catch (const Error& e) {
    huv::set_last_error(e.what());
    return e.status;
  }
}

huv_status huv_plan_describe(void* plan, char* buf, int32_t capacity) {
  if (!plan || !buf || capacity <= 0) return HUV_ERR_INVALID_PARAMETER;
  const std::string& r = static_cast<Plan*>(plan)->report;
  std::strncpy(buf, r.c_str(), static_cast<size_t>(capacity) - 1);
  buf[capacity - 1] = 0;
  return static_cast<int32_t>(r.size()) < capacity ? HUV_OK : HUV_ERR_DIMENSION_MISMATCH;
}

void huv_plan_destroy(void* plan) { delete static_cast<Plan*>(plan); }

}  // extern "C"
