// tm_batch.cu -- batches of (image, template[, mask]) pairs: one persistent
// tensor-core launch per group of compatible pairs, CUDA graphs, autotuning.
//
// The reference matches one pair per call (src/template_matching.rs:78, :125)
// and finds extremes in a second pass (:479-511). Here a batch is planned once:
//   * every pair is checked with the reference's assertions, in order;
//   * a kernel family is chosen per pair: tcgen05 tensor cores where the
//     template shape allows, else the CUDA-core exact kernel (or the
//     reference-order kernel for REFERENCE_F32); the autotuner can time both
//     on the first pair of each shape class and keep the faster;
//   * tensor-core pairs are grouped by tensor-memory row width and mask
//     kind; the autotuner times each group's launch with its natural row
//     width or twice it and each tile height, and groups that end on the
//     same (width, height, mask kind) merge; each runs as ONE persistent
//     launch over all its tiles with find_extremes fused into the epilogue;
//   * the extremes keys are armed at creation and re-armed by the finish
//     kernel, so a launch is the group kernels plus one finish kernel;
//   * the groups' launches run side by side on two streams, the group with
//     the longest tiles first, each claiming tiles from its own counter, so
//     the SMs that one launch leaves idle in its last wave take tiles of the
//     next instead of waiting for the slowest CTA;
//   * the launch sequence is captured once in a CUDA graph and replayed.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "tm_common.cuh"
#include "tm_internal.h"

#define IPB_API extern "C" __attribute__((visibility("default")))

struct ipb_batch_plan {
  int device = -1;
  int precision = 0;
  std::vector<ipb::MatchArgs> args;  // per pair, device pointers
  std::vector<ipb_extremes_f32*> ext_out;
  std::vector<bool> tensor;
  std::vector<unsigned long long*> key_of;  // fused extremes keys per pair, or null
  struct Group {
    ipb::UmmaPlan plan;
    std::vector<uint32_t> members;
    std::vector<ipb::UmmaProblem> probs;
    ipb::UmmaProblem* d_probs = nullptr;
    uint32_t tiles = 0;
  };
  std::vector<Group> groups;
  // unmasked pairs of one template on the row-operand kernel: up to 8 per
  // launch, with the template blocks and window sums in the group's scratch
  struct RowGroup {
    std::vector<uint32_t> members;
    void* d_scratch = nullptr;
  };
  std::vector<RowGroup> rgroups;
  // fused extremes of tensor pairs: keys {min, max}, map widths, output records
  unsigned long long* d_keys = nullptr;
  uint32_t* d_widths = nullptr;
  ipb_extremes_f32** d_outs = nullptr;
  uint32_t nkeys = 0;
  // CUDA-core pairs: scratch and extremes scratch
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  void* d_ext_scratch = nullptr;
  ipb::ExtremesResult<float>* d_ext_result = nullptr;
  unsigned int* d_err = nullptr;
  unsigned int tag = 0;
  // tile counters of the groups' launches (two words each) and, with two or
  // more groups, the stream and events the later groups run on
  unsigned int* d_sched = nullptr;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  uint32_t kernels = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace ipb {
namespace {

// ---- autotuner -----------------------------------------------------------------
// Two decisions are tuned and cached per process, and persisted in a text file
// (IPB_TUNING_FILE, default ~/.cache/imageproc_b200/tuning.txt; an empty
// IPB_TUNING_FILE keeps them in memory only):
//  * per batch group (on unless IPB_AUTOTUNE=0): the tensor-memory row width
//    (the group's natural width or twice it) and the tile height, timed on
//    the group's own pairs; key = (natural width, masked, tallest template
//    rounded up to 8, log2 of the group's output positions, log2 of its
//    largest image side). Line: "group ks0 masked h8 wlog mlog ks nt".
//  * per pair shape class (IPB_AUTOTUNE=1): tensor cores or the CUDA-core
//    kernel, timed on the first pair of each (w, h, masked, normalised).
//    Line: "pair w h masked norm tensor".
struct TuneKey {
  uint32_t w, h;
  int masked, norm;
  bool operator<(const TuneKey& o) const {
    return std::tie(w, h, masked, norm) < std::tie(o.w, o.h, o.masked, o.norm);
  }
};
struct GroupKey {
  uint32_t ks0;
  int masked;
  uint32_t h8, wlog, mlog, set;
  bool operator<(const GroupKey& o) const {
    return std::tie(ks0, masked, h8, wlog, mlog, set) < std::tie(o.ks0, o.masked, o.h8, o.wlog, o.mlog, o.set);
  }
};
struct GroupChoice {
  uint32_t ks, nt, set;
};
std::mutex g_tune_mu;
std::map<TuneKey, bool> g_tune;
std::map<GroupKey, GroupChoice> g_group_tune;
bool g_tune_loaded = false;

std::string tuning_file() {
  const char* f = std::getenv("IPB_TUNING_FILE");
  if (f) return f;
  const char* home = std::getenv("HOME");
  if (!home || !*home) return "";
  const std::string dir = std::string(home) + "/.cache/imageproc_b200";
  mkdir((std::string(home) + "/.cache").c_str(), 0755);
  mkdir(dir.c_str(), 0755);
  return dir + "/tuning.txt";
}

void tune_load_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const std::string f = tuning_file();
  if (f.empty()) return;
  std::ifstream in(f);
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string kind;
    ls >> kind;
    if (kind == "pair") {
      TuneKey k;
      int t;
      if (ls >> k.w >> k.h >> k.masked >> k.norm >> t) g_tune[k] = t != 0;
    } else if (kind == "group2") {
      GroupKey k;
      GroupChoice c;
      if (ls >> k.ks0 >> k.masked >> k.h8 >> k.wlog >> k.mlog >> k.set >> c.ks >> c.nt >> c.set && c.set >= 1 &&
          c.set <= kMaxSet)
        g_group_tune[k] = c;
    }
  }
}

void tune_store_locked() {
  const std::string f = tuning_file();
  if (f.empty()) return;
  const std::string tmp = f + ".tmp" + std::to_string((long)getpid());
  {
    std::ofstream out(tmp);
    for (auto& kv : g_tune)
      out << "pair " << kv.first.w << ' ' << kv.first.h << ' ' << kv.first.masked << ' ' << kv.first.norm << ' '
          << (kv.second ? 1 : 0) << '\n';
    for (auto& kv : g_group_tune)
      out << "group2 " << kv.first.ks0 << ' ' << kv.first.masked << ' ' << kv.first.h8 << ' ' << kv.first.wlog
          << ' ' << kv.first.mlog << ' ' << kv.first.set << ' ' << kv.second.ks << ' ' << kv.second.nt << ' '
          << kv.second.set << '\n';
    if (!out) return;
  }
  std::rename(tmp.c_str(), f.c_str());  // whole files only, for processes sharing the file
}

// Largest set of pairs sharing an image that a launch computes together
// (IPB_SET_MAX = 1..4; default 4; 1 computes every pair alone).
uint32_t set_cap() {
  const char* v = std::getenv("IPB_SET_MAX");
  const int n = v ? std::atoi(v) : (int)kMaxSet;
  return n < 1 ? 1u : (n > (int)kMaxSet ? kMaxSet : (uint32_t)n);
}

int autotune_mode() {  // 0: off, 1: groups, 2: groups and per-pair paths
  const char* v = std::getenv("IPB_AUTOTUNE");
  if (!v) return 1;
  if (std::strcmp(v, "0") == 0) return 0;
  if (std::strcmp(v, "1") == 0) return 2;
  return 1;
}

uint32_t floor_log2(double v) {
  uint32_t l = 0;
  while (v >= 2.0) {
    v *= 0.5;
    ++l;
  }
  return l;
}

// Cost model: tensor cores whenever the shape is supported (they win from
// 16x8 templates up; below that the CUDA-core kernel takes the pair).
bool model_prefers_tensor(const MatchArgs& a) { return umma_supported(a); }

float time_launch(const MatchArgs& a, bool tensor, void* scratch, unsigned int* err) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, a.stream);
    if (tensor) launch_umma(a, err, 0);
    else launch_exact_cc(a, scratch);
    cudaEventRecord(e1, a.stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

bool choose_tensor(const MatchArgs& a, bool autotune, void* scratch, unsigned int* err) {
  if (!umma_supported(a)) return false;
  const int path = kernel_path();
  if (path == 1) return false;
  if (path == 2 || !autotune) return model_prefers_tensor(a);
  const TuneKey k{a.w, a.h, a.mask ? 1 : 0, method_is_norm(a.method) ? 1 : 0};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(k);
    if (it != g_tune.end()) return it->second;
  }
  const float tt = time_launch(a, true, scratch, err);
  const float tc = time_launch(a, false, scratch, err);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[k] = tt <= tc;
  tune_store_locked();
  return tt <= tc;
}

ipb_status to_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IPB_OK;
  const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  (void)cudaGetLastError();
  return (ipb_status)report_error(e == cudaErrorMemoryAllocation ? IPB_ERR_OUT_OF_MEMORY : IPB_ERR_CUDA,
                                  msg.c_str());
}

#define IPB_TRY(call, what)                           \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return to_status(e_, what); \
  } while (0)

// Times a natural group's launch with each candidate (row width ks0 or
// 2 ks0, each tile height) on the group's own pairs and returns the fastest.
// The timing launches write the pairs' outputs and extremes keys; the
// caller re-arms the keys afterwards.
template <class KeysOf>
ipb_status tune_group(ipb_batch_plan* p, const std::vector<uint32_t>& mem, uint32_t ks0, bool masked, uint32_t hmax,
                      uint32_t set, KeysOf keys_of, GroupChoice& best) {
  best = GroupChoice{ks0, 0, 1};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  IPB_TRY(cudaEventCreate(&e0), "event");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return to_status(cudaErrorMemoryAllocation, "event");
  }
  float best_ms = 1e30f;
  cudaError_t err = cudaSuccess;
  // sets of 1, 2 and the largest the pairs form; each with its tile heights
  std::vector<uint32_t> sets{1u};
  if (set >= 2) sets.push_back(2u);
  if (set > 2) sets.push_back(set);
  for (uint32_t ks : {ks0, 2 * ks0}) {
   for (uint32_t sz : sets) {
    uint32_t nts[2];
    const uint32_t nnt = umma_tile_heights(masked, sz, nts);
    for (uint32_t t = 0; t < nnt && err == cudaSuccess; ++t) {
      UmmaPlan pl;
      if (!umma_plan_for(ks, masked, hmax, pl, nts[t], sz)) continue;
      std::vector<UmmaProblem> probs;
      for (uint32_t i : mem) probs.push_back(umma_problem(p->args[i], pl, 0, keys_of(i)));
      const uint32_t tiles = umma_make_sets(probs, pl);
      UmmaLaunch L{};
      UmmaProblem* d_probs = nullptr;
      if (probs.size() > kInlineProblems) {
        if ((err = cudaMalloc(&d_probs, sizeof(UmmaProblem) * probs.size())) != cudaSuccess) break;
        cudaMemcpy(d_probs, probs.data(), sizeof(UmmaProblem) * probs.size(), cudaMemcpyHostToDevice);
      } else {
        for (size_t i = 0; i < probs.size(); ++i) L.inl[i] = probs[i];
      }
      L.probs = d_probs;
      L.nprobs = (uint32_t)probs.size();
      L.tiles = tiles;
      L.err = p->d_err;
      L.tag = p->tag;
      L.wait_ns = pipeline_wait_ns();
      L.stall = 0u;
      L.sched = p->d_sched;
      float ms_best = 1e30f;
      for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) {  // the first launch is a warm-up
        cudaEventRecord(e0, nullptr);
        err = launch_umma_batch(pl, L, nullptr, nullptr);
        cudaEventRecord(e1, nullptr);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0;
        if (err == cudaSuccess && rep > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
          ms_best = std::min(ms_best, ms);
      }
      if (d_probs) cudaFree(d_probs);
      if (err == cudaSuccess && ms_best < best_ms) {
        best_ms = ms_best;
        best = GroupChoice{ks, nts[t], sz};
      }
    }
   }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return to_status(err, "tuning launch");
}

void release(ipb_batch_plan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  for (auto& g : p->groups)
    if (g.d_probs) cudaFree(g.d_probs);
  for (auto& g : p->rgroups)
    if (g.d_scratch) cudaFree(g.d_scratch);
  for (void* b : {(void*)p->d_keys, (void*)p->d_widths, (void*)p->d_outs, p->d_scratch, p->d_ext_scratch,
                  (void*)p->d_ext_result, (void*)p->d_err, (void*)p->d_sched})
    if (b) cudaFree(b);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  if (p->side) cudaStreamDestroy(p->side);
}

// Enqueue the plan's launch sequence (used once under stream capture, and
// directly when profiling so each kernel can be timed).
ipb_status enqueue(ipb_batch_plan* p, cudaStream_t s, bool timed, uint32_t* kernels) {
  uint32_t k = 0;  // the keys were armed at creation and are re-armed by the finish kernel
  // groups after the first run on the side stream, between a fork and a join
  // on s; concurrent launches are timed as one span on s
  const bool side_by_side = p->groups.size() + p->rgroups.size() >= 2 && p->side;
  KernelTimer* span = timed && side_by_side ? acquire_kernel_timer() : nullptr;
  double span_macs = 0, span_bytes = 0;
  if (span) {
    timer_begin(span, kKernelUmma, s);
    span->launches = (uint32_t)p->groups.size();
  }
  if (side_by_side) {
    IPB_TRY(cudaEventRecord(p->ev_fork, s), "fork");
    IPB_TRY(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "fork");
  }
  cudaError_t launch_err = cudaSuccess;
  for (size_t gi = 0; gi < p->groups.size(); ++gi) {
    const ipb_batch_plan::Group& g = p->groups[gi];
    const cudaStream_t gs = side_by_side && gi > 0 ? p->side : s;
    UmmaLaunch L{};
    const uint32_t n = (uint32_t)g.probs.size();
    if (n <= kInlineProblems)
      for (uint32_t i = 0; i < n; ++i) L.inl[i] = g.probs[i];
    L.probs = g.d_probs;
    L.nprobs = n;
    L.tiles = g.tiles;
    L.err = p->d_err;
    L.tag = p->tag;
    L.wait_ns = pipeline_wait_ns();
    L.stall = pipeline_stall() ? 1u : 0u;
    L.sched = p->d_sched + 2 * gi;
    KernelTimer* t = timed && !side_by_side ? acquire_kernel_timer() : nullptr;
    launch_err = launch_umma_batch(g.plan, L, gs, t);
    if (launch_err != cudaSuccess) break;
    double macs = 0, bytes = 0;
    for (uint32_t i : g.members) {
      const MatchArgs& a = p->args[i];
      const double Wo = a.W - a.w + 1.0, Ho = a.H - a.h + 1.0, tp = (double)a.w * a.h;
      macs += Wo * Ho * tp;
      bytes += (double)a.W * a.H + tp * (a.mask ? 2.0 : 1.0) + 4.0 * Wo * Ho;
    }
    if (t) note_kernel_timed(t, macs, bytes);
    span_macs += macs;
    span_bytes += bytes;
    ++k;
  }
  for (size_t ri = 0; ri < p->rgroups.size() && launch_err == cudaSuccess; ++ri) {
    const ipb_batch_plan::RowGroup& g = p->rgroups[ri];
    const cudaStream_t gs = side_by_side && (ri > 0 || !p->groups.empty()) ? p->side : s;
    std::vector<MatchArgs> probs;
    std::vector<unsigned long long*> ext;
    double macs = 0, bytes = 0;
    for (uint32_t i : g.members) {
      probs.push_back(p->args[i]);
      ext.push_back(p->key_of[i]);
      const MatchArgs& a = p->args[i];
      const double Wo = a.W - a.w + 1.0, Ho = a.H - a.h + 1.0, tp = (double)a.w * a.h;
      macs += Wo * Ho * tp;
      bytes += (double)a.W * a.H + tp + 4.0 * Wo * Ho;
    }
    KernelTimer* t = timed && !side_by_side ? acquire_kernel_timer() : nullptr;
    launch_err = launch_shift_multi(probs.data(), ext.data(), (uint32_t)probs.size(), g.d_scratch, p->d_err,
                                    p->tag, gs, t);
    if (launch_err != cudaSuccess) break;
    if (t) note_kernel_timed(t, macs, bytes);
    span_macs += macs;
    span_bytes += bytes;
    // template blocks, one window-sum map per image, the matching launch
    std::vector<const uint8_t*> imgs;
    for (const MatchArgs& a : probs)
      if (a.method != IPB_CROSS_CORRELATION && std::find(imgs.begin(), imgs.end(), a.img) == imgs.end())
        imgs.push_back(a.img);
    k += 2 + (uint32_t)imgs.size();
  }
  if (side_by_side) {
    // joined on every path, a failed launch included, so that s orders all of
    // the side stream's work before the caller's next use of it
    IPB_TRY(cudaEventRecord(p->ev_join, p->side), "join");
    IPB_TRY(cudaStreamWaitEvent(s, p->ev_join, 0), "join");
  }
  IPB_TRY(launch_err, "tensor-core batch launch");
  if (span) {
    timer_end(span, s);
    note_kernel_timed(span, span_macs, span_bytes);
  }
  for (size_t i = 0; i < p->args.size(); ++i) {
    if (p->tensor[i]) continue;
    MatchArgs a = p->args[i];
    a.stream = s;
    if (a.w == 0 || a.h == 0) {
      IPB_TRY(cudaMemsetAsync(a.out, 0, (size_t)(a.W - a.w + 1) * (a.H - a.h + 1) * sizeof(float), s), "memset");
    } else if (a.precision == IPB_PRECISION_REFERENCE_F32) {
      IPB_TRY(launch_reference(a, p->d_scratch), "reference launch");
      k += 2;
    } else {
      IPB_TRY(launch_exact_cc(a, p->d_scratch), "CUDA-core launch");
      k += (!a.mask && a.method != IPB_CROSS_CORRELATION) ? 4 : 2;
    }
    if (p->ext_out[i]) {
      IPB_TRY(launch_find_extremes<float>(a.out, (unsigned long long)(a.W - a.w + 1) * (a.H - a.h + 1),
                                          p->d_ext_scratch, p->d_ext_result, s),
              "find_extremes launch");
      IPB_TRY(launch_extremes_to_struct(p->d_ext_result, a.W - a.w + 1, p->ext_out[i], s), "extremes record");
      k += 2;
    }
  }
  if (p->nkeys) {
    IPB_TRY(launch_extremes_keys_finish(p->d_keys, p->d_widths, p->d_outs, p->nkeys, s), "extremes finish");
    ++k;
  }
  if (kernels) *kernels = k;
  return IPB_OK;
}

ipb_status create(const ipb_pair* pairs, uint32_t n, int precision, bool capture, ipb_batch_plan** out) {
  if (!out || (n && !pairs)) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null argument");
  if (precision < 0 || precision > 2) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "unknown precision");
  for (uint32_t i = 0; i < n; ++i) {
    const ipb_pair& q = pairs[i];
    const int st = check_match_args(q.image_width, q.image_height, q.template_width, q.template_height,
                                     q.mask != nullptr, q.mask_width, q.mask_height, q.method);
    if (st != IPB_OK) {
      std::string msg = std::string("pair ") + std::to_string(i) + ": " + ipb_last_error_message();
      return (ipb_status)report_error(st, msg.c_str());
    }
    if (!q.out || (!q.image && (size_t)q.image_width * q.image_height) ||
        (!q.templ && (size_t)q.template_width * q.template_height))
      return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, ("pair " + std::to_string(i) + ": null buffer").c_str());
  }
  auto* p = new ipb_batch_plan();
  cudaGetDevice(&p->device);
  p->precision = precision;
  p->args.resize(n);
  p->ext_out.resize(n);
  p->tensor.assign(n, false);
  size_t scratch = 256;
  for (uint32_t i = 0; i < n; ++i) {
    const ipb_pair& q = pairs[i];
    MatchArgs a{q.image, q.image_width, q.image_height, q.templ, q.template_width, q.template_height,
                q.mask, q.mask && q.mask_is_binary != 0, q.method, precision, q.out, nullptr};
    p->args[i] = a;
    p->ext_out[i] = q.extremes;
    if (a.w && a.h)
      scratch = std::max(scratch, precision == IPB_PRECISION_REFERENCE_F32 ? reference_scratch_bytes(a)
                                                                           : exact_cc_scratch_bytes(a));
  }
  auto fail = [&](ipb_status st) {
    release(p);
    delete p;
    return st;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&p->d_scratch, scratch)) != cudaSuccess) return fail(to_status(e, "cudaMalloc"));
  p->scratch_bytes = scratch;
  if ((e = cudaMalloc(&p->d_err, sizeof(unsigned int))) != cudaSuccess) return fail(to_status(e, "cudaMalloc"));
  cudaMemset(p->d_err, 0, sizeof(unsigned int));
  if ((e = cudaMalloc(&p->d_ext_scratch, extremes_scratch_bytes())) != cudaSuccess)
    return fail(to_status(e, "cudaMalloc"));
  cudaMemset(p->d_ext_scratch, 0, extremes_scratch_bytes());
  if ((e = cudaMalloc(&p->d_ext_result, sizeof(ExtremesResult<float>))) != cudaSuccess)
    return fail(to_status(e, "cudaMalloc"));

  // kernel family per pair, then tensor groups keyed by (row width, masked)
  const int tune = autotune_mode();
  std::map<uint32_t, std::vector<uint32_t>> by_key;
  // unmasked pairs the row-operand kernel takes, by template (pointer and size)
  std::map<std::tuple<const uint8_t*, uint32_t, uint32_t>, std::vector<uint32_t>> by_tpl;
  for (uint32_t i = 0; i < n; ++i) {
    MatchArgs a = p->args[i];
    if (!a.w || !a.h) continue;
    a.stream = nullptr;
    if (shift_preferred(a)) {
      p->tensor[i] = true;
      by_tpl[std::make_tuple(a.tpl, a.w, a.h)].push_back(i);
      continue;
    }
    if (choose_tensor(a, tune == 2, p->d_scratch, p->d_err)) {
      p->tensor[i] = true;
      by_key[umma_group_key(a)].push_back(i);
    }
  }
  std::vector<uint32_t> widths;
  std::vector<ipb_extremes_f32*> outs;
  // one key slot per tensor pair with an extremes record
  std::vector<int> slot(n, -1);
  for (uint32_t i = 0; i < n; ++i)
    if (p->tensor[i] && p->ext_out[i]) {
      slot[i] = (int)widths.size();
      widths.push_back(p->args[i].W - p->args[i].w + 1);
      outs.push_back(p->ext_out[i]);
    }
  p->nkeys = (uint32_t)widths.size();
  if (p->nkeys) {
    if ((e = cudaMalloc(&p->d_keys, sizeof(unsigned long long) * 2 * p->nkeys)) != cudaSuccess ||
        (e = cudaMalloc(&p->d_widths, sizeof(uint32_t) * p->nkeys)) != cudaSuccess ||
        (e = cudaMalloc(&p->d_outs, sizeof(void*) * p->nkeys)) != cudaSuccess)
      return fail(to_status(e, "cudaMalloc"));
    cudaMemcpy(p->d_widths, widths.data(), sizeof(uint32_t) * p->nkeys, cudaMemcpyHostToDevice);
    cudaMemcpy(p->d_outs, outs.data(), sizeof(void*) * p->nkeys, cudaMemcpyHostToDevice);
  }
  if ((e = umma_prepare_kernels()) != cudaSuccess) return fail(to_status(e, "kernel attributes"));
  if (!by_key.empty()) {
    // tile counters: two words per launch, reset by each launch's last CTA
    const size_t sched_bytes = sizeof(unsigned int) * 2 * by_key.size();
    if ((e = cudaMalloc(&p->d_sched, sched_bytes)) != cudaSuccess) return fail(to_status(e, "cudaMalloc"));
    if ((e = cudaMemset(p->d_sched, 0, sched_bytes)) != cudaSuccess) return fail(to_status(e, "cudaMemset"));
  }
  auto keys_of = [&](uint32_t i) { return slot[i] >= 0 ? p->d_keys + 2 * slot[i] : nullptr; };
  p->key_of.resize(n);
  for (uint32_t i = 0; i < n; ++i) p->key_of[i] = keys_of(i);
  for (auto& kv : by_tpl)
    for (size_t b = 0; b < kv.second.size(); b += kShiftMaxProblems) {
      ipb_batch_plan::RowGroup g;
      g.members.assign(kv.second.begin() + b,
                       kv.second.begin() + std::min(kv.second.size(), b + (size_t)kShiftMaxProblems));
      std::vector<MatchArgs> probs;
      for (uint32_t i : g.members) probs.push_back(p->args[i]);
      if ((e = cudaMalloc(&g.d_scratch, shift_multi_scratch_bytes(probs.data(), (uint32_t)probs.size()))) !=
          cudaSuccess)
        return fail(to_status(e, "cudaMalloc"));
      p->rgroups.push_back(std::move(g));
    }
  // the largest set the pairs `mem` form (pairs on one image with one
  // template size), within the set cap
  auto set_of = [&](const std::vector<uint32_t>& mem) {
    std::vector<UmmaProblem> probs;
    UmmaPlan any{};
    for (uint32_t i : mem) probs.push_back(umma_problem(p->args[i], any, 0, nullptr));
    return std::max(1u, std::min(umma_largest_set(probs), set_cap()));
  };
  // each natural group's (row width, tile height): tuned, or the natural
  // width with the tallest tiles; groups that land on the same (width,
  // height, mask kind) share one launch
  std::map<std::tuple<bool, uint32_t, uint32_t, uint32_t>, std::vector<uint32_t>> launches;
  for (auto& kv : by_key) {
    const std::vector<uint32_t>& mem = kv.second;
    const bool masked = p->args[mem.front()].mask != nullptr;
    const uint32_t ks0 = kv.first / 2;  // umma_group_key = row width * 2 + masked
    const uint32_t set = set_of(mem);
    // untuned: sets of up to four unmasked pairs, two binary-mask pairs
    GroupChoice c{ks0, 0, masked ? std::min(set, 2u) : set};
    if (tune) {
      uint32_t hmax = 0, side = 0;
      double pos = 0;
      for (uint32_t i : mem) {
        const MatchArgs& a = p->args[i];
        hmax = std::max(hmax, a.h);
        side = std::max(side, std::max(a.W, a.H));
        pos += (double)(a.W - a.w + 1) * (a.H - a.h + 1);
      }
      const GroupKey gk{ks0, masked ? 1 : 0, (hmax + 7) & ~7u, floor_log2(pos), floor_log2(side), set};
      bool have = false;
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_load_locked();
        auto it = g_group_tune.find(gk);
        if (it != g_group_tune.end()) {
          c = it->second;
          have = true;
        }
      }
      if (!have) {
        ipb_status st = tune_group(p, mem, ks0, masked, hmax, set, keys_of, c);
        if (st != IPB_OK) return fail(st);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_group_tune[gk] = c;
        tune_store_locked();
      }
    }
    auto& dst = launches[std::make_tuple(masked, c.ks, c.nt, c.set)];
    dst.insert(dst.end(), mem.begin(), mem.end());
  }
  for (auto& kv : launches) {
    ipb_batch_plan::Group g;
    const bool masked = std::get<0>(kv.first);
    uint32_t ks = std::get<1>(kv.first);
    const uint32_t nt = std::get<2>(kv.first);
    g.members = kv.second;
    std::sort(g.members.begin(), g.members.end());
    uint32_t hmax = 0;
    for (uint32_t i : g.members) {
      hmax = std::max(hmax, p->args[i].h);
      ks = std::max(ks, umma_row_width(p->args[i].w));
    }
    // a cached choice that no longer fits falls back to the tallest tiles,
    // then to problems alone
    const uint32_t set = std::min(std::get<3>(kv.first), set_of(g.members));
    if (!umma_plan_for(ks, masked, hmax, g.plan, nt, set) && !umma_plan_for(ks, masked, hmax, g.plan, 0, set) &&
        !umma_plan_for(ks, masked, hmax, g.plan, 0, 1))
      return fail((ipb_status)report_error(IPB_ERR_CUDA, "no tensor-core plan"));
    for (uint32_t i : g.members) g.probs.push_back(umma_problem(p->args[i], g.plan, 0, keys_of(i)));
    g.tiles = umma_make_sets(g.probs, g.plan);
    if (g.probs.size() > kInlineProblems) {
      if ((e = cudaMalloc(&g.d_probs, sizeof(UmmaProblem) * g.probs.size())) != cudaSuccess)
        return fail(to_status(e, "cudaMalloc"));
      cudaMemcpy(g.d_probs, g.probs.data(), sizeof(UmmaProblem) * g.probs.size(), cudaMemcpyHostToDevice);
    }
    p->groups.push_back(std::move(g));
  }
  // arm the extremes keys (after any tuning launches) and clear the error word
  if (p->nkeys && ((e = launch_extremes_keys_init(p->d_keys, p->nkeys, nullptr)) != cudaSuccess ||
                   (e = cudaStreamSynchronize(nullptr)) != cudaSuccess))
    return fail(to_status(e, "extremes keys"));
  if ((e = cudaMemset(p->d_err, 0, sizeof(unsigned int))) != cudaSuccess) return fail(to_status(e, "cudaMemset"));
  // longest tiles first (binary masks: three correlations per row; then the
  // widest rows), so that the launch started second fills the tail of the first
  std::stable_sort(p->groups.begin(), p->groups.end(),
                   [](const ipb_batch_plan::Group& x, const ipb_batch_plan::Group& y) {
                     if (x.plan.masked != y.plan.masked) return x.plan.masked;
                     return x.plan.ks > y.plan.ks;
                   });
  if (p->groups.size() + p->rgroups.size() >= 2) {
    if ((e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming)) != cudaSuccess)
      return fail(to_status(e, "side stream"));
  }
  uint32_t kernels = 0;
  if (capture) {
    // capture the launch sequence once
    cudaStream_t cs;
    if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess)
      return fail(to_status(e, "stream"));
    ipb_status st = IPB_OK;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      st = enqueue(p, cs, false, &kernels);
      cudaGraph_t graph = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
      if (st == IPB_OK && e2 == cudaSuccess) {
        p->graph = graph;
        e = cudaGraphInstantiate(&p->exec, graph, 0);
      } else if (e2 != cudaSuccess) {
        e = e2;
      }
    }
    cudaStreamDestroy(cs);
    if (st != IPB_OK) return fail(st);
    if (e != cudaSuccess) return fail(to_status(e, "graph capture"));
    p->kernels = kernels;
  }
  *out = p;
  return IPB_OK;
}

}  // namespace
}  // namespace ipb

using namespace ipb;

IPB_API ipb_status ipb_batch_plan_create(const ipb_pair* pairs, uint32_t n, int precision, ipb_batch_plan** plan) {
  return create(pairs, n, precision, /*capture=*/true, plan);
}

IPB_API ipb_status ipb_batch_plan_launch(ipb_batch_plan* plan, void* stream) {
  if (!plan) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (profiling_enabled()) return enqueue(plan, s, true, nullptr);  // timed kernels, no graph
  cudaError_t e = cudaGraphLaunch(plan->exec, s);
  if (e != cudaSuccess) return to_status(e, "cudaGraphLaunch");
  count_launches(plan->kernels);
  return IPB_OK;
}

IPB_API ipb_status ipb_batch_plan_info(const ipb_batch_plan* plan, uint32_t* kernels, uint32_t* tensor_pairs) {
  if (!plan) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null plan");
  if (kernels) *kernels = plan->kernels;
  if (tensor_pairs) *tensor_pairs = (uint32_t)std::count(plan->tensor.begin(), plan->tensor.end(), true);
  return IPB_OK;
}

IPB_API void ipb_batch_tuning_reset(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  g_group_tune.clear();
  g_tune_loaded = false;
}

IPB_API ipb_status ipb_batch_plan_groups(const ipb_batch_plan* plan, uint32_t max, ipb_batch_group* out,
                                         uint32_t* count) {
  if (!plan || (max && !out)) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null argument");
  const uint32_t n = (uint32_t)plan->groups.size();
  for (uint32_t i = 0; i < n && i < max; ++i) {
    const ipb_batch_plan::Group& g = plan->groups[i];
    out[i] = ipb_batch_group{g.plan.ks, g.plan.NT, g.plan.masked ? 1 : 0, (uint32_t)g.members.size(), g.tiles,
                             g.plan.set_max};
  }
  if (count) *count = n;
  return IPB_OK;
}

IPB_API ipb_status ipb_batch_plan_destroy(ipb_batch_plan* plan) {
  if (!plan) return IPB_OK;
  cudaDeviceSynchronize();
  release(plan);
  delete plan;
  return IPB_OK;
}

IPB_API ipb_status ipb_match_template_batch_device(const ipb_pair* pairs, uint32_t n, int precision,
                                                   void* stream) {
  ipb_batch_plan* p = nullptr;
  ipb_status st = create(pairs, n, precision, /*capture=*/false, &p);
  if (st != IPB_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = enqueue(p, s, profiling_enabled(), nullptr);
  // the plan's descriptors and scratch must outlive the enqueued work
  const cudaError_t e = cudaStreamSynchronize(s);
  release(p);
  delete p;
  if (st != IPB_OK) return st;
  return to_status(e, "cudaStreamSynchronize");
}
