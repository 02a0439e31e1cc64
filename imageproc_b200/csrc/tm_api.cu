// tm_api.cu -- the C ABI (include/imageproc_b200.h): argument checks, device
// memory, streams and dispatch to the kernels.
//
// Each calling thread owns one context per device: a stream for the
// host-pointer entry points, grow-only device buffers, and an event marking the
// last use of its scratch memory. Every call waits for that event on its own
// stream before touching scratch and records it afterwards, so calls from one
// thread on different streams never overlap on shared scratch.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <thread>
#include <deque>
#include <map>
#include <mutex>
#include <vector>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>

#include "tm_common.cuh"
#include "tm_internal.h"

#define IPB_API extern "C" __attribute__((visibility("default")))

namespace ipb {

// ---- tracing ----------------------------------------------------------------
namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned long long> g_launches_by_kernel[kKernelCount];
std::atomic<bool> g_profiling{false};

struct TimedLaunch {
  KernelTimer timer;
  double macs, bytes;
};
struct KernelStats {
  unsigned long long launches = 0;
  double ms = 0, macs = 0, bytes = 0;
};
std::mutex g_prof_mu;
std::deque<TimedLaunch> g_pending;         // recorded, not yet collected (stable addresses)
std::vector<KernelTimer> g_free_timers;    // event pairs for reuse
KernelStats g_stats[kKernelCount];

void settle_pending_locked() {
  for (TimedLaunch& t : g_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.timer.end) == cudaSuccess &&
        cudaEventElapsedTime(&ms, t.timer.begin, t.timer.end) == cudaSuccess && t.timer.kernel >= 0) {
      KernelStats& k = g_stats[t.timer.kernel];
      k.launches += t.timer.launches;
      k.ms += ms;
      k.macs += t.macs;
      k.bytes += t.bytes;
    }
    g_free_timers.push_back(t.timer);
  }
  g_pending.clear();
}

KernelTimer* acquire_timer() {
  if (!g_profiling.load()) return nullptr;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (g_pending.size() > 4096) settle_pending_locked();
  KernelTimer t;
  if (!g_free_timers.empty()) {
    t = g_free_timers.back();
    g_free_timers.pop_back();
  } else if (cudaEventCreate(&t.begin) != cudaSuccess || cudaEventCreate(&t.end) != cudaSuccess) {
    return nullptr;
  }
  t.kernel = -1;
  t.launches = 1;
  g_pending.push_back({t, 0.0, 0.0});
  return &g_pending.back().timer;
}

void note_timed(KernelTimer* t, double macs, double bytes) {
  if (!t) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto it = g_pending.rbegin(); it != g_pending.rend(); ++it)
    if (&it->timer == t) {
      it->macs = macs;
      it->bytes = bytes;
      return;
    }
}
}  // namespace

const char* kernel_name(int id) {
  static const char* names[kKernelCount] = {
      "template_prep", "integral_rows", "integral_cols", "exact_cc",
      "template_sum_f32", "reference_f32", "find_extremes", "umma_i8", "many_i8", "suppress", "filter",
      "example", "proposal_net", "propose", "rows_i8", "window_sq_sums"};
  return id >= 0 && id < kKernelCount ? names[id] : "unknown";
}

void count_launch(int id) {
  g_launches.fetch_add(1);
  if (id >= 0 && id < kKernelCount) g_launches_by_kernel[id].fetch_add(1);
}

namespace {
std::atomic<unsigned long long> g_wait_ns{kDefaultWaitNs};
}  // namespace

unsigned long long pipeline_wait_ns() { return g_wait_ns.load(std::memory_order_relaxed); }
namespace {
std::atomic<bool> g_stall{false};
}  // namespace
bool pipeline_stall() { return g_stall.load(std::memory_order_relaxed); }

int device_sm_count() {
  static std::atomic<int> cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev >= 0 && dev < 64) {
    const int n = cache[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
  }
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  if (dev >= 0 && dev < 64) cache[dev].store(n, std::memory_order_relaxed);
  return n;
}

namespace {

thread_local std::string g_last_error;

int precision_from_env() {
  const char* v = std::getenv("IPB_PRECISION");
  if (!v) return IPB_PRECISION_EXACT_FP64;
  if (!std::strcmp(v, "1") || !std::strcmp(v, "exact_f32")) return IPB_PRECISION_EXACT_F32;
  if (!std::strcmp(v, "2") || !std::strcmp(v, "reference_f32")) return IPB_PRECISION_REFERENCE_F32;
  return IPB_PRECISION_EXACT_FP64;
}
std::atomic<int> g_precision{precision_from_env()};

// Kernel family for exact matches: 0 = choose (tensor cores where the shape
// allows), 1 = CUDA cores only, 2 = tensor cores wherever supported (the
// Hankel-row kernel), 3 = the row-operand tensor kernel wherever it applies.
int path_from_env() {
  const char* v = std::getenv("IPB_PATH");
  if (!v) return 0;
  if (!std::strcmp(v, "1") || !std::strcmp(v, "cuda_core")) return 1;
  if (!std::strcmp(v, "2") || !std::strcmp(v, "tensor")) return 2;
  if (!std::strcmp(v, "3") || !std::strcmp(v, "row_operand")) return 3;
  return 0;
}
std::atomic<int> g_path{path_from_env()};

// Row bands of the host-buffer match calls: 0 = choose from the map's size,
// n >= 1 = n bands (tuning).
int bands_from_env() {
  const char* v = std::getenv("IPB_HOST_BANDS");
  if (!v) return 0;
  const int n = std::atoi(v);
  return n < 0 ? 0 : n;
}
const int g_host_bands = bands_from_env();
constexpr uint32_t kMaxBands = 16;

ipb_status fail(ipb_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

ipb_status cuda_fail(cudaError_t e, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  (void)cudaGetLastError();  // clear a sticky non-fatal error so the next call starts clean
  if (e == cudaErrorMemoryAllocation) return fail(IPB_ERR_OUT_OF_MEMORY, msg);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(IPB_ERR_NO_DEVICE, msg);
  return fail(IPB_ERR_CUDA, msg);
}

#define IPB_CUDA(call, what)                         \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t last = nullptr;  // last use of any scratch buffer below
  DevBuf scratch, ext_scratch, ext_result, img, tpl, mask, out;
  void* pinned = nullptr;  // small pinned host block: reduction results, error words
  DevBuf errw;                     // tensor-core error word (largest failing launch tag)
  DevBuf many_keys;                // per-template extremes keys of the many-templates path
  DevBuf rgb, keys;                // the example workflow: RGB canvas, score-map range
  unsigned int tag = 0;            // tag of the last tensor-core launch
  unsigned int tag_checked = 0;    // largest failing tag already reported
  bool tensor_since_check = false;
  // copy streams of the banded host calls: image rows in, score rows out;
  // tensor-core bands run on streams of their own
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaStream_t s_band[kMaxBands] = {};
  cudaEvent_t band_in[kMaxBands] = {}, band_done[kMaxBands] = {}, out_done = nullptr;
  // page-locked bounce buffer for pageable images of banded calls; free for
  // reuse once stage_free (recorded after its last copy) has completed
  void* stage = nullptr;
  size_t stage_cap = 0;
  cudaEvent_t stage_free = nullptr;
  // page-locked bounce buffer for pageable score maps of banded calls: each
  // band's rows land there and the host copies them out while later bands
  // are still computed and copied (band_out[b]: band b's rows have landed)
  void* ostage = nullptr;
  size_t ostage_cap = 0;
  cudaEvent_t band_out[kMaxBands] = {};
  ~Context() {
    if (device < 0) return;
    cudaSetDevice(device);
    if (last) cudaEventSynchronize(last);
    for (cudaStream_t s : {s_in, s_out})
      if (s) cudaStreamSynchronize(s);
    for (uint32_t b = 0; b < kMaxBands; ++b) {
      if (s_band[b]) {
        cudaStreamSynchronize(s_band[b]);
        cudaStreamDestroy(s_band[b]);
      }
      if (band_in[b]) cudaEventDestroy(band_in[b]);
      if (band_done[b]) cudaEventDestroy(band_done[b]);
      if (band_out[b]) cudaEventDestroy(band_out[b]);
    }
    if (out_done) cudaEventDestroy(out_done);
    if (stage_free) {
      cudaEventSynchronize(stage_free);
      cudaEventDestroy(stage_free);
    }
    if (stage) cudaFreeHost(stage);
    if (ostage) cudaFreeHost(ostage);
    for (cudaStream_t s : {s_in, s_out})
      if (s) cudaStreamDestroy(s);
    for (DevBuf* b : {&scratch, &ext_scratch, &ext_result, &img, &tpl, &mask, &out, &errw, &many_keys, &rgb, &keys})
      if (b->p) cudaFree(b->p);
    if (pinned) cudaFreeHost(pinned);
    if (last) cudaEventDestroy(last);
    if (stream) cudaStreamDestroy(stream);
  }
};

ipb_status get_ctx(Context** out) {
  thread_local std::unordered_map<int, std::unique_ptr<Context>> ctxs;
  int dev = 0;
  IPB_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  auto it = ctxs.find(dev);
  if (it != ctxs.end()) {
    *out = it->second.get();
    return IPB_OK;
  }
  cudaDeviceProp prop;
  IPB_CUDA(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  if (prop.major != 10)
    return fail(IPB_ERR_NO_DEVICE, std::string("imageproc_b200 needs an sm_100 (B200) device; device ") +
                                       std::to_string(dev) + " is " + prop.name);
  auto c = std::make_unique<Context>();
  c->device = dev;
  IPB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  IPB_CUDA(cudaEventCreateWithFlags(&c->last, cudaEventDisableTiming), "cudaEventCreate");
  IPB_CUDA(cudaMallocHost(&c->pinned, 256), "cudaMallocHost");
  *out = c.get();
  ctxs.emplace(dev, std::move(c));
  return IPB_OK;
}

// Grow-only device buffer. The old block may still be read by queued work, so
// wait for the context's last recorded use before freeing it.
ipb_status ensure(Context* c, DevBuf& b, size_t bytes, bool zero = false) {
  if (bytes == 0) bytes = 1;
  if (b.cap >= bytes) return IPB_OK;
  IPB_CUDA(cudaEventSynchronize(c->last), "cudaEventSynchronize");
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  }
  const size_t cap = align_up(bytes, 1 << 20);
  IPB_CUDA(cudaMalloc(&b.p, cap), "cudaMalloc");
  b.cap = cap;
  if (zero) IPB_CUDA(cudaMemset(b.p, 0, cap), "cudaMemset");
  return IPB_OK;
}

// The reference's assertions, in its order: ImageTemplateMask::new checks the
// mask first (:433-437), then ImageTemplate::new checks width and height
// (:395-402).
ipb_status check_match(uint32_t W, uint32_t H, uint32_t w, uint32_t h, bool masked, uint32_t mw,
                       uint32_t mh, int method) {
  if (masked && (mw != w || mh != h))
    return fail(IPB_ERR_MASK_SIZE, "the template and mask must be the same size");
  if (W < w) return fail(IPB_ERR_TEMPLATE_WIDTH, "image width must be greater than or equal to template width");
  if (H < h)
    return fail(IPB_ERR_TEMPLATE_HEIGHT, "image height must be greater than or equal to template height");
  if (method < 0 || method > 3) return fail(IPB_ERR_INVALID_ARGUMENT, "unknown MatchTemplateMethod");
  return IPB_OK;
}

bool host_mask_is_binary(const uint8_t* m, size_t n) {
  for (size_t k = 0; k < n; ++k)
    if (m[k] > 1) return false;
  return true;
}

// Synchronises the stream and reports a tensor-core wait that ran out in any
// launch of this context since the last check (the error word holds the
// largest failing launch tag; tags only grow).
ipb_status finish_sync(Context* c, cudaStream_t s) {
  const bool check = c->tensor_since_check && c->errw.p;
  if (check)
    IPB_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(c->pinned) + 128, c->errw.p, sizeof(unsigned int),
                             cudaMemcpyDeviceToHost, s),
             "copy error word");
  IPB_CUDA(cudaEventRecord(c->last, s), "cudaEventRecord");
  IPB_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (check) {
    c->tensor_since_check = false;
    const unsigned int failed = *reinterpret_cast<volatile unsigned int*>(static_cast<uint8_t*>(c->pinned) + 128);
    if (failed > c->tag_checked) {
      c->tag_checked = failed;
      return fail(IPB_ERR_TIMEOUT, "a tensor-core template-matching kernel timed out waiting on its pipeline");
    }
  }
  return IPB_OK;
}

// Enqueue one matching problem on a.stream.
ipb_status run_match(Context* c, const MatchArgs& a) {
  const size_t out_bytes = (size_t)(a.W - a.w + 1) * (a.H - a.h + 1) * sizeof(float);
  if (a.w == 0 || a.h == 0) {
    // empty window: every score is 0 (the walk never runs, :410-416)
    IPB_CUDA(cudaMemsetAsync(a.out, 0, out_bytes, a.stream), "cudaMemsetAsync");
    return IPB_OK;
  }
  const bool ref = a.precision == IPB_PRECISION_REFERENCE_F32;
  const int path = g_path.load();
  const bool rows = !ref && path == 3 && shift_supported(a);
  const bool tensor = !ref && !rows && path != 1 && umma_supported(a);
  ipb_status st;
  if (rows) {
    if ((st = ensure(c, c->errw, sizeof(unsigned int), /*zero=*/true)) ||
        (st = ensure(c, c->scratch, shift_scratch_bytes(a))))
      return st;
  } else if (tensor) {
    if ((st = ensure(c, c->errw, sizeof(unsigned int), /*zero=*/true))) return st;
  } else {
    const size_t need = ref ? reference_scratch_bytes(a) : exact_cc_scratch_bytes(a);
    if ((st = ensure(c, c->scratch, need))) return st;
  }
  IPB_CUDA(cudaStreamWaitEvent(a.stream, c->last, 0), "cudaStreamWaitEvent");
  MatchArgs la = a;
  la.timer = acquire_timer();
  cudaError_t e;
  if (rows) {
    c->tag += 1;
    c->tensor_since_check = true;
    e = launch_shift(la, c->scratch.p, nullptr, static_cast<unsigned int*>(c->errw.p), c->tag);
  } else if (tensor) {
    c->tag += 1;
    c->tensor_since_check = true;
    e = launch_umma(la, static_cast<unsigned int*>(c->errw.p), c->tag);
  } else {
    e = ref ? launch_reference(la, c->scratch.p) : launch_exact_cc(la, c->scratch.p);
  }
  if (la.timer) {
    const double Wo = a.W - a.w + 1.0, Ho = a.H - a.h + 1.0, tp = (double)a.w * a.h;
    note_timed(la.timer, Wo * Ho * tp,
               (double)a.W * a.H + tp * (a.mask ? 2.0 : 1.0) + 4.0 * Wo * Ho);
  }
  if (e != cudaSuccess) return cuda_fail(e, "template-matching launch");
  IPB_CUDA(cudaEventRecord(c->last, a.stream), "cudaEventRecord");
  return IPB_OK;
}

// How many row bands a host-buffer match is cut into. One call moves the
// image in, computes and moves the map out; in bands the three overlap (image
// rows of band b+1 cross PCIe while band b is scored and band b-1's scores
// come back), so the call costs about its larger copy instead of the sum.
// A map below 2 MiB is one band: its copies are shorter than a launch.
uint32_t host_bands(size_t out_bytes, uint32_t Ho, uint32_t w, uint32_t h) {
  if (w == 0 || h == 0) return 1;
  uint32_t n = g_host_bands > 0 ? (uint32_t)g_host_bands : (out_bytes >= (4u << 20) ? 4u : out_bytes >= (2u << 20) ? 2u : 1u);
  n = std::min(n, kMaxBands);
  return std::min(n, (Ho + 15) / 16);  // bands of at least 16 score rows
}

ipb_status ensure_band_streams(Context* c, uint32_t nb) {
  for (cudaStream_t* s : {&c->s_in, &c->s_out})
    if (!*s) IPB_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "cudaStreamCreate");
  for (uint32_t b = 0; b < nb; ++b)
    if (!c->s_band[b]) IPB_CUDA(cudaStreamCreateWithFlags(&c->s_band[b], cudaStreamNonBlocking), "cudaStreamCreate");
  for (uint32_t b = 0; b < kMaxBands; ++b) {
    if (!c->band_in[b]) IPB_CUDA(cudaEventCreateWithFlags(&c->band_in[b], cudaEventDisableTiming), "cudaEventCreate");
    if (!c->band_done[b])
      IPB_CUDA(cudaEventCreateWithFlags(&c->band_done[b], cudaEventDisableTiming), "cudaEventCreate");
    if (!c->band_out[b])
      IPB_CUDA(cudaEventCreateWithFlags(&c->band_out[b], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (!c->out_done) IPB_CUDA(cudaEventCreateWithFlags(&c->out_done, cudaEventDisableTiming), "cudaEventCreate");
  return IPB_OK;
}

// The host-buffer match in nb row bands. Band b scores rows [o0, o1) of the
// map from image rows [o0, o1 + h - 1): a problem of its own whose output
// rows keep the full map's pitch, so every score is the one the whole-map
// launch writes. Image rows cross once, in order (a band copies only the rows
// the previous band did not); bands start on multiples of 16 rows so a
// 16-byte-aligned image stays aligned. A band is under one wave of SMs, so
// a launch of it takes about as long as the whole map's: tensor-core bands
// therefore run on streams of their own, each starting once its image rows
// are in, beside the bands before it (they share no scratch). CUDA-core bands
// share the context's scratch and run in order on the context's stream.
// Host-to-host copies split over a few persistent threads (the calling
// thread takes a share too). A pageable source cannot be read by the copy
// engines directly: the driver would stage it through its own buffer at one
// thread's memcpy rate while holding the calling thread. Copying it into a
// page-locked buffer in parallel, band by band, lets each band's DMA start
// while the next band's rows are still being copied. The workers spin on the
// job generation for a short while after their last job (calls come in
// bursts; a sleeping thread takes tens of microseconds to wake), then sleep
// on a condition variable. One batch of jobs at a time.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool;
    return pool;
  }
  void copy(uint8_t* dst, const uint8_t* src, size_t n) {
    const size_t parts = (n >= (size_t(1) << 18) && !workers_.empty()) ? workers_.size() + 1 : 1;
    if (parts == 1) {
      std::memcpy(dst, src, n);
      return;
    }
    std::lock_guard<std::mutex> batch(batch_mu_);
    const size_t chunk = align_up((n + parts - 1) / parts, 4096);
    uint32_t nj = 0;
    for (size_t off = chunk; off < n && nj < kMaxJobs; off += chunk)
      jobs_[nj++] = Job{dst + off, src + off, std::min(chunk, n - off)};
    njobs_.store(nj, std::memory_order_relaxed);
    pending_.store(nj, std::memory_order_relaxed);
    const uint64_t g = ++gen_;
    // publishes the jobs: a claim carries its batch's generation, so a worker
    // still holding an older generation takes nothing from this batch
    claim_.store(g << 32, std::memory_order_release);
    if (sleepers_.load(std::memory_order_acquire) > 0) {
      std::lock_guard<std::mutex> lk(mu_);
      cv_.notify_all();
    }
    std::memcpy(dst, src, std::min(chunk, n));
    run_jobs(g);  // help with what the workers have not taken yet
    while (pending_.load(std::memory_order_acquire) != 0) {
    }
  }
  ~CopyPool() {
    stop_.store(true, std::memory_order_release);
    {
      std::lock_guard<std::mutex> lk(mu_);
      cv_.notify_all();
    }
    for (std::thread& t : workers_) t.join();
  }

 private:
  struct Job {
    uint8_t* dst;
    const uint8_t* src;
    size_t n;
  };
  static constexpr uint32_t kMaxJobs = 8;
  CopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = hw >= 8 ? 3u : (hw >= 4 ? 1u : 0u);
    for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this] { run(); });
  }
  // Takes jobs of batch g until none is left (or a newer batch replaced it).
  void run_jobs(uint64_t g) {
    uint64_t c = claim_.load(std::memory_order_acquire);
    for (;;) {
      if ((c >> 32) != g || (uint32_t)c >= njobs_.load(std::memory_order_relaxed)) return;
      if (!claim_.compare_exchange_weak(c, c + 1, std::memory_order_acq_rel, std::memory_order_acquire)) continue;
      const Job& j = jobs_[(uint32_t)c];
      std::memcpy(j.dst, j.src, j.n);
      pending_.fetch_sub(1, std::memory_order_release);
      c = claim_.load(std::memory_order_acquire);
    }
  }
  void run() {
    uint64_t seen = 0;
    while (!stop_.load(std::memory_order_acquire)) {
      const auto spin_until = std::chrono::steady_clock::now() + std::chrono::microseconds(500);
      uint64_t g = claim_.load(std::memory_order_acquire) >> 32;
      while (g == seen && !stop_.load(std::memory_order_relaxed) && std::chrono::steady_clock::now() < spin_until)
        g = claim_.load(std::memory_order_acquire) >> 32;
      if (g == seen) {
        std::unique_lock<std::mutex> lk(mu_);
        sleepers_.fetch_add(1, std::memory_order_acq_rel);
        cv_.wait(lk, [&] {
          return stop_.load(std::memory_order_acquire) || (claim_.load(std::memory_order_acquire) >> 32) != seen;
        });
        sleepers_.fetch_sub(1, std::memory_order_acq_rel);
        continue;
      }
      seen = g;
      run_jobs(g);
    }
  }
  std::mutex batch_mu_, mu_;
  std::condition_variable cv_;
  Job jobs_[kMaxJobs];
  std::atomic<uint32_t> njobs_{0};
  uint64_t gen_ = 0;
  std::atomic<uint64_t> claim_{0};  // generation << 32 | next job
  std::atomic<uint32_t> pending_{0}, sleepers_{0};
  std::atomic<bool> stop_{false};
  std::vector<std::thread> workers_;
};

bool host_memory_is_locked(const void* p) {
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, p) == cudaSuccess) return pa.type == cudaMemoryTypeHost;
  (void)cudaGetLastError();  // not a pointer the runtime knows: pageable
  return false;
}

ipb_status host_match_banded(Context* c, const MatchArgs& full, const uint8_t* image, const uint8_t* tpl,
                             const uint8_t* mask, uint32_t nb, float* out) {
  ipb_status st;
  if ((st = ensure_band_streams(c, nb))) return st;
  const int path = g_path.load();
  const bool side_by_side =
      full.precision != IPB_PRECISION_REFERENCE_F32 && path != 1 && path != 3 && umma_supported(full);
  if (side_by_side && (st = ensure(c, c->errw, sizeof(unsigned int), /*zero=*/true))) return st;
  // A copy into page-locked memory returns at once, so a band's score rows are
  // queued as soon as its launch is: they cross while the host still copies
  // later image rows. A pageable score map is reached through the output
  // bounce buffer, which the host drains band by band at the end.
  const bool out_locked = host_memory_is_locked(out);
  const uint32_t W = full.W, Wo = full.W - full.w + 1, Ho = full.H - full.h + 1;
  // a pageable image goes through the context's page-locked bounce buffer
  const size_t ib = (size_t)W * full.H;
  const bool staged = ib >= (size_t(1) << 20) && !host_memory_is_locked(image);
  if (staged) {
    if (c->stage_free) IPB_CUDA(cudaEventSynchronize(c->stage_free), "cudaEventSynchronize");
    if (c->stage_cap < ib) {
      if (c->stage) cudaFreeHost(c->stage);
      c->stage = nullptr;
      c->stage_cap = 0;
      IPB_CUDA(cudaMallocHost(&c->stage, align_up(ib, 1 << 20)), "cudaMallocHost (image staging)");
      c->stage_cap = align_up(ib, 1 << 20);
    }
    if (!c->stage_free) IPB_CUDA(cudaEventCreateWithFlags(&c->stage_free, cudaEventDisableTiming), "cudaEventCreate");
  }
  // a pageable score map goes through the page-locked output bounce buffer
  const size_t ob = (size_t)Wo * Ho * sizeof(float);
  const bool ostaged = !out_locked && ob > 0;
  if (ostaged && c->ostage_cap < ob) {
    if (c->ostage) cudaFreeHost(c->ostage);
    c->ostage = nullptr;
    c->ostage_cap = 0;
    IPB_CUDA(cudaMallocHost(&c->ostage, align_up(ob, 1 << 20)), "cudaMallocHost (score staging)");
    c->ostage_cap = align_up(ob, 1 << 20);
  }
  float* dst_out = ostaged ? static_cast<float*>(c->ostage) : out;
  const uint8_t* src_img = staged ? static_cast<const uint8_t*>(c->stage) : image;
  const size_t tb = (size_t)full.w * full.h;
  const uint32_t rows = (uint32_t)align_up((Ho + nb - 1) / nb, 16);
  uint8_t* d_img = static_cast<uint8_t*>(c->img.p);
  auto queue_out = [&](uint32_t b) -> ipb_status {
    const uint32_t o0 = b * rows, o1 = std::min(Ho, o0 + rows);
    IPB_CUDA(cudaStreamWaitEvent(c->s_out, c->band_done[b], 0), "cudaStreamWaitEvent");
    IPB_CUDA(cudaMemcpyAsync(dst_out + (size_t)o0 * Wo, full.out + (size_t)o0 * Wo,
                             (size_t)(o1 - o0) * Wo * sizeof(float), cudaMemcpyDeviceToHost, c->s_out),
             "copy score rows");
    IPB_CUDA(cudaEventRecord(c->band_out[b], c->s_out), "cudaEventRecord");
    return IPB_OK;
  };
  auto enqueue = [&]() -> ipb_status {
    IPB_CUDA(cudaStreamWaitEvent(c->s_in, c->last, 0), "cudaStreamWaitEvent");
    IPB_CUDA(cudaMemcpyAsync(c->tpl.p, tpl, tb, cudaMemcpyHostToDevice, c->s_in), "copy template");
    if (mask) IPB_CUDA(cudaMemcpyAsync(c->mask.p, mask, tb, cudaMemcpyHostToDevice, c->s_in), "copy mask");
    uint32_t have = 0, bands = 0;  // image rows on the device, bands queued
    for (uint32_t o0 = 0; o0 < Ho; o0 += rows, ++bands) {
      const uint32_t o1 = std::min(Ho, o0 + rows), need = o1 + full.h - 1;
      if (staged)
        CopyPool::get().copy(static_cast<uint8_t*>(c->stage) + (size_t)have * W, image + (size_t)have * W,
                             (size_t)(need - have) * W);
      IPB_CUDA(cudaMemcpyAsync(d_img + (size_t)have * W, src_img + (size_t)have * W, (size_t)(need - have) * W,
                               cudaMemcpyHostToDevice, c->s_in),
               "copy image rows");
      have = need;
      IPB_CUDA(cudaEventRecord(c->band_in[bands], c->s_in), "cudaEventRecord");
      MatchArgs a = full;
      a.img = full.img + (size_t)o0 * W;
      a.H = need - o0;
      a.out = full.out + (size_t)o0 * Wo;
      if (side_by_side) {
        a.stream = c->s_band[bands];
        IPB_CUDA(cudaStreamWaitEvent(a.stream, c->band_in[bands], 0), "cudaStreamWaitEvent");
        a.timer = acquire_timer();
        c->tag += 1;
        c->tensor_since_check = true;
        const cudaError_t e = launch_umma(a, static_cast<unsigned int*>(c->errw.p), c->tag);
        if (a.timer) {
          const double tp = (double)a.w * a.h, Ho_b = a.H - a.h + 1.0;
          note_timed(a.timer, Wo * Ho_b * tp, (double)a.W * a.H + tp * (a.mask ? 2.0 : 1.0) + 4.0 * Wo * Ho_b);
        }
        if (e != cudaSuccess) return cuda_fail(e, "template-matching launch");
      } else {
        IPB_CUDA(cudaStreamWaitEvent(c->stream, c->band_in[bands], 0), "cudaStreamWaitEvent");
        ipb_status s2 = run_match(c, a);
        if (s2) return s2;
      }
      IPB_CUDA(cudaEventRecord(c->band_done[bands], a.stream), "cudaEventRecord");
      if ((st = queue_out(bands))) return st;
    }
    if (staged) IPB_CUDA(cudaEventRecord(c->stage_free, c->s_in), "cudaEventRecord");
    IPB_CUDA(cudaEventRecord(c->out_done, c->s_out), "cudaEventRecord");
    IPB_CUDA(cudaStreamWaitEvent(c->stream, c->out_done, 0), "cudaStreamWaitEvent");
    if (ostaged)
      // each band's rows to the caller's buffer as soon as they have landed,
      // while later bands are still in flight
      for (uint32_t b = 0; b < bands; ++b) {
        IPB_CUDA(cudaEventSynchronize(c->band_out[b]), "cudaEventSynchronize");
        const uint32_t o0 = b * rows, o1 = std::min(Ho, o0 + rows);
        CopyPool::get().copy(reinterpret_cast<uint8_t*>(out + (size_t)o0 * Wo),
                             reinterpret_cast<const uint8_t*>(dst_out + (size_t)o0 * Wo),
                             (size_t)(o1 - o0) * Wo * sizeof(float));
      }
    return IPB_OK;
  };
  if ((st = enqueue())) {
    // nothing may touch the caller's buffers after the call returns
    cudaStreamSynchronize(c->s_in);
    cudaStreamSynchronize(c->stream);
    for (uint32_t b = 0; b < nb; ++b) cudaStreamSynchronize(c->s_band[b]);
    cudaStreamSynchronize(c->s_out);
    return st;
  }
  return finish_sync(c, c->stream);
}

ipb_status host_match(const uint8_t* image, uint32_t W, uint32_t H, const uint8_t* tpl, uint32_t w,
                      uint32_t h, int method, const uint8_t* mask, uint32_t mw, uint32_t mh,
                      float* out) {
  ipb_status st = check_match(W, H, w, h, mask != nullptr, mw, mh, method);
  if (st) return st;
  if ((!image && (size_t)W * H) || (!tpl && (size_t)w * h) || !out)
    return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  const size_t ib = (size_t)W * H, tb = (size_t)w * h;
  const size_t ob = (size_t)(W - w + 1) * (H - h + 1) * sizeof(float);
  if ((st = ensure(c, c->img, ib)) || (st = ensure(c, c->tpl, tb)) || (st = ensure(c, c->out, ob)))
    return st;
  if (mask && (st = ensure(c, c->mask, tb))) return st;
  MatchArgs a{static_cast<const uint8_t*>(c->img.p), W, H, static_cast<const uint8_t*>(c->tpl.p), w, h,
              mask ? static_cast<const uint8_t*>(c->mask.p) : nullptr,
              mask ? host_mask_is_binary(mask, tb) : false, method, g_precision.load(),
              static_cast<float*>(c->out.p), c->stream};
  const uint32_t nb = host_bands(ob, H - h + 1, w, h);
  if (nb > 1) return host_match_banded(c, a, image, tpl, mask, nb, out);
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  if (ib) IPB_CUDA(cudaMemcpyAsync(c->img.p, image, ib, cudaMemcpyHostToDevice, c->stream), "copy image");
  if (tb) IPB_CUDA(cudaMemcpyAsync(c->tpl.p, tpl, tb, cudaMemcpyHostToDevice, c->stream), "copy template");
  if (mask && tb)
    IPB_CUDA(cudaMemcpyAsync(c->mask.p, mask, tb, cudaMemcpyHostToDevice, c->stream), "copy mask");
  if ((st = run_match(c, a))) return st;
  IPB_CUDA(cudaMemcpyAsync(out, c->out.p, ob, cudaMemcpyDeviceToHost, c->stream), "copy scores");
  return finish_sync(c, c->stream);
}

template <typename T, typename R>
ipb_status extremes_common(Context* c, const T* d, uint32_t W, uint32_t H, R* out, cudaStream_t s) {
  using DT = typename std::conditional<
      std::is_same<T, uint64_t>::value, unsigned long long,
      typename std::conditional<std::is_same<T, int64_t>::value, long long, T>::type>::type;
  ipb_status st;
  if ((st = ensure(c, c->ext_scratch, extremes_scratch_bytes(), /*zero=*/true))) return st;
  if ((st = ensure(c, c->ext_result, sizeof(ExtremesResult<DT>)))) return st;
  IPB_CUDA(cudaStreamWaitEvent(s, c->last, 0), "cudaStreamWaitEvent");
  auto* res = static_cast<ExtremesResult<DT>*>(c->ext_result.p);
  cudaError_t e = launch_find_extremes<DT>(reinterpret_cast<const DT*>(d), (unsigned long long)W * H,
                                           c->ext_scratch.p, res, s);
  if (e != cudaSuccess) return cuda_fail(e, "find_extremes launch");
  IPB_CUDA(cudaMemcpyAsync(c->pinned, res, sizeof(ExtremesResult<DT>), cudaMemcpyDeviceToHost, s),
           "copy extremes");
  if ((st = finish_sync(c, s))) return st;
  ExtremesResult<DT> r;
  std::memcpy(&r, c->pinned, sizeof(r));
  out->max_value = (T)r.max_value;
  out->min_value = (T)r.min_value;
  out->max_value_location_x = (uint32_t)(r.max_index % W);
  out->max_value_location_y = (uint32_t)(r.max_index / W);
  out->min_value_location_x = (uint32_t)(r.min_index % W);
  out->min_value_location_y = (uint32_t)(r.min_index / W);
  return IPB_OK;
}

template <typename T, typename R>
ipb_status extremes_host(const T* image, uint32_t W, uint32_t H, R* out) {
  if (W == 0 || H == 0) return fail(IPB_ERR_EMPTY_IMAGE, "image must be non-empty");
  if (!image || !out) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  const size_t bytes = (size_t)W * H * sizeof(T);
  if ((st = ensure(c, c->img, bytes))) return st;
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(cudaMemcpyAsync(c->img.p, image, bytes, cudaMemcpyHostToDevice, c->stream), "copy image");
  return extremes_common<T, R>(c, static_cast<const T*>(c->img.p), W, H, out, c->stream);
}

template <typename T, typename R>
ipb_status extremes_device(const T* d_image, uint32_t W, uint32_t H, R* out, void* stream) {
  if (W == 0 || H == 0) return fail(IPB_ERR_EMPTY_IMAGE, "image must be non-empty");
  if (!d_image || !out) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  return extremes_common<T, R>(c, d_image, W, H, out, static_cast<cudaStream_t>(stream));
}

}  // namespace

int report_error(int st, const char* msg) { return fail(static_cast<ipb_status>(st), msg); }

int check_match_args(uint32_t W, uint32_t H, uint32_t w, uint32_t h, bool masked, uint32_t mw, uint32_t mh,
                     int method) {
  return check_match(W, H, w, h, masked, mw, mh, method);
}

void count_launches(unsigned long long n) { g_launches.fetch_add(n); }
bool profiling_enabled() { return g_profiling.load(); }
KernelTimer* acquire_kernel_timer() { return acquire_timer(); }
void note_kernel_timed(KernelTimer* t, double macs, double bytes) { note_timed(t, macs, bytes); }
int kernel_path() { return g_path.load(); }

}  // namespace ipb

using namespace ipb;

IPB_API const char* ipb_last_error_message(void) { return g_last_error.c_str(); }

IPB_API const char* ipb_version(void) { return "imageproc_b200 0.1.0 (sm_100a)"; }

// ---- page-locked host buffers ---------------------------------------------------
namespace {
std::mutex g_host_mu;
std::unordered_map<void*, size_t> g_host_live;  // pointer -> block size
std::multimap<size_t, void*> g_host_free;        // cached blocks by size
size_t g_host_cached = 0;
constexpr size_t kHostCacheMax = size_t(1) << 30;
}  // namespace

IPB_API void* ipb_host_alloc(size_t bytes) {
  const size_t sz = align_up(bytes ? bytes : 1, size_t(1) << 16);
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    auto it = g_host_free.lower_bound(sz);
    if (it != g_host_free.end() && it->first <= 2 * sz) {  // reuse a block at most twice the size
      void* p = it->second;
      g_host_cached -= it->first;
      g_host_live[p] = it->first;
      g_host_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaHostAlloc(&p, sz, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_host_mu);
  g_host_live[p] = sz;
  return p;
}

IPB_API void ipb_host_free(void* ptr) {
  if (!ptr) return;
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    auto it = g_host_live.find(ptr);
    if (it == g_host_live.end()) return;  // not a block of this cache
    const size_t sz = it->second;
    g_host_live.erase(it);
    if (g_host_cached + sz <= kHostCacheMax) {
      g_host_free.emplace(sz, ptr);
      g_host_cached += sz;
      return;
    }
  }
  cudaFreeHost(ptr);
}

IPB_API void ipb_host_cache_release(void) {
  std::multimap<size_t, void*> blocks;
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    blocks.swap(g_host_free);
    g_host_cached = 0;
  }
  for (auto& kv : blocks) cudaFreeHost(kv.second);
}

IPB_API uint64_t ipb_launch_count(void) { return g_launches.load(); }

IPB_API ipb_status ipb_profile_enable(int enable) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  settle_pending_locked();
  g_profiling.store(enable != 0);
  return IPB_OK;
}

IPB_API int ipb_profile_collect(ipb_kernel_stats* out, int max_entries) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  settle_pending_locked();
  int n = 0;
  for (int k = 0; k < kKernelCount; ++k) {
    if (!g_stats[k].launches) continue;
    if (out && n < max_entries) {
      out[n].name = kernel_name(k);
      out[n].launches = g_stats[k].launches;
      out[n].total_ms = g_stats[k].ms;
      out[n].algorithmic_macs = g_stats[k].macs;
      out[n].algorithmic_bytes = g_stats[k].bytes;
    }
    ++n;
    g_stats[k] = KernelStats{};
  }
  return n;
}

IPB_API ipb_status ipb_set_precision(int precision) {
  if (precision < 0 || precision > 2) return fail(IPB_ERR_INVALID_ARGUMENT, "unknown precision");
  g_precision.store(precision);
  return IPB_OK;
}

IPB_API int ipb_get_precision(void) { return g_precision.load(); }

IPB_API void ipb_debug_stall_pipelines(int enable) { g_stall.store(enable != 0, std::memory_order_relaxed); }

IPB_API void ipb_debug_set_pipeline_wait_ns(uint64_t ns) {
  g_wait_ns.store(ns ? (unsigned long long)ns : kDefaultWaitNs, std::memory_order_relaxed);
}

IPB_API ipb_status ipb_set_path(int path) {
  if (path < 0 || path > 3) return fail(IPB_ERR_INVALID_ARGUMENT, "unknown kernel path");
  g_path.store(path);
  return IPB_OK;
}

IPB_API int ipb_get_path(void) { return g_path.load(); }

IPB_API ipb_status ipb_match_template(const uint8_t* image, uint32_t W, uint32_t H, const uint8_t* tpl,
                                      uint32_t w, uint32_t h, int method, float* out) {
  return host_match(image, W, H, tpl, w, h, method, nullptr, 0, 0, out);
}

IPB_API ipb_status ipb_match_template_parallel(const uint8_t* image, uint32_t W, uint32_t H,
                                               const uint8_t* tpl, uint32_t w, uint32_t h, int method,
                                               float* out) {
  return host_match(image, W, H, tpl, w, h, method, nullptr, 0, 0, out);
}

IPB_API ipb_status ipb_match_template_with_mask(const uint8_t* image, uint32_t W, uint32_t H,
                                                const uint8_t* tpl, uint32_t w, uint32_t h, int method,
                                                const uint8_t* mask, uint32_t mw, uint32_t mh,
                                                float* out) {
  if (!mask) return fail(IPB_ERR_INVALID_ARGUMENT, "null mask");
  return host_match(image, W, H, tpl, w, h, method, mask, mw, mh, out);
}

IPB_API ipb_status ipb_match_template_with_mask_parallel(const uint8_t* image, uint32_t W, uint32_t H,
                                                         const uint8_t* tpl, uint32_t w, uint32_t h,
                                                         int method, const uint8_t* mask, uint32_t mw,
                                                         uint32_t mh, float* out) {
  if (!mask) return fail(IPB_ERR_INVALID_ARGUMENT, "null mask");
  return host_match(image, W, H, tpl, w, h, method, mask, mw, mh, out);
}

IPB_API ipb_status ipb_match_templates_device(const uint8_t* d_image, uint32_t W, uint32_t H,
                                              const uint8_t* d_templates, uint32_t w, uint32_t h, uint32_t n,
                                              int method, int precision, float* d_out,
                                              ipb_extremes_f32* d_extremes, void* stream) {
  ipb_status st = check_match(W, H, w, h, false, 0, 0, method);
  if (st) return st;
  if (precision < 0 || precision > 2) return fail(IPB_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!many_supported(w, h, n, precision))
    return fail(IPB_ERR_INVALID_ARGUMENT,
                "ipb_match_templates_device takes 16..64 x 1..64 templates in an exact precision; use "
                "ipb_match_template_batch_device for other shapes");
  if (!d_image || !d_templates || (!d_out && !d_extremes)) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  if (d_extremes && (uint64_t)(W - w + 1) * (H - h + 1) > 0xFFFFFFFFull)
    return fail(IPB_ERR_INVALID_ARGUMENT, "fused extremes take score maps of fewer than 2^32 positions");
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  if ((st = ensure(c, c->errw, sizeof(unsigned int), /*zero=*/true))) return st;
  if (d_extremes && (st = ensure(c, c->many_keys, sizeof(unsigned long long) * 2 * n))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  IPB_CUDA(cudaStreamWaitEvent(s, c->last, 0), "cudaStreamWaitEvent");
  unsigned long long* keys = d_extremes ? static_cast<unsigned long long*>(c->many_keys.p) : nullptr;
  if (keys) IPB_CUDA(launch_many_keys_init(keys, n, s), "extremes init");
  c->tag += 1;
  c->tensor_since_check = true;
  KernelTimer* t = acquire_timer();
  const cudaError_t e = launch_many(d_image, W, H, d_templates, w, h, n, method, precision, d_out, keys,
                                    static_cast<unsigned int*>(c->errw.p), c->tag, s, t);
  if (t) {
    const double Wo = W - w + 1.0, Ho = H - h + 1.0, tp = (double)w * h;
    note_timed(t, Wo * Ho * tp * n, (double)W * H + tp * n + (d_out ? 4.0 * Wo * Ho * n : 0.0));
  }
  if (e != cudaSuccess) return cuda_fail(e, "many-templates launch");
  if (keys) IPB_CUDA(launch_many_keys_finish(keys, W - w + 1, d_extremes, n, s), "extremes finish");
  IPB_CUDA(cudaEventRecord(c->last, s), "cudaEventRecord");
  return IPB_OK;
}

// ---- integral images -------------------------------------------------------------
namespace {
ipb_status check_sat_args(uint32_t channels, int bits) {
  if (channels != 1 && channels != 3 && channels != 4)
    return fail(IPB_ERR_INVALID_ARGUMENT, "channels must be 1 (Luma), 3 (Rgb) or 4 (Rgba)");
  if (bits != 32 && bits != 64) return fail(IPB_ERR_INVALID_ARGUMENT, "integral images are u32 or u64");
  return IPB_OK;
}

ipb_status host_sat(const uint8_t* image, uint32_t W, uint32_t H, uint32_t channels, bool squared, int bits,
                    void* out) {
  ipb_status st = check_sat_args(channels, bits);
  if (st) return st;
  const size_t ib = (size_t)W * H * channels;
  const size_t ob = (size_t)(W + 1) * (H + 1) * channels * (bits / 8);
  if ((!image && ib) || !out) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  if ((st = ensure(c, c->img, ib)) || (st = ensure(c, c->out, ob))) return st;
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  if (ib) IPB_CUDA(cudaMemcpyAsync(c->img.p, image, ib, cudaMemcpyHostToDevice, c->stream), "copy image");
  IPB_CUDA(launch_sat(static_cast<const uint8_t*>(c->img.p), W, H, channels, squared, bits, c->out.p, c->stream),
           "integral image launch");
  IPB_CUDA(cudaMemcpyAsync(out, c->out.p, ob, cudaMemcpyDeviceToHost, c->stream), "copy integral image");
  return finish_sync(c, c->stream);
}
}  // namespace

IPB_API ipb_status ipb_integral_image_u32(const uint8_t* image, uint32_t W, uint32_t H, uint32_t channels,
                                          uint32_t* out) {
  return host_sat(image, W, H, channels, false, 32, out);
}
IPB_API ipb_status ipb_integral_squared_image_u32(const uint8_t* image, uint32_t W, uint32_t H,
                                                  uint32_t channels, uint32_t* out) {
  return host_sat(image, W, H, channels, true, 32, out);
}
IPB_API ipb_status ipb_integral_image_u64(const uint8_t* image, uint32_t W, uint32_t H, uint32_t channels,
                                          uint64_t* out) {
  return host_sat(image, W, H, channels, false, 64, out);
}
IPB_API ipb_status ipb_integral_squared_image_u64(const uint8_t* image, uint32_t W, uint32_t H,
                                                  uint32_t channels, uint64_t* out) {
  return host_sat(image, W, H, channels, true, 64, out);
}
IPB_API ipb_status ipb_integral_image_device(const uint8_t* d_image, uint32_t W, uint32_t H, uint32_t channels,
                                             int squared, int bits, void* d_out, void* stream) {
  ipb_status st = check_sat_args(channels, bits);
  if (st) return st;
  if ((!d_image && (size_t)W * H) || !d_out) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  IPB_CUDA(launch_sat(d_image, W, H, channels, squared != 0, bits, d_out, static_cast<cudaStream_t>(stream)),
           "integral image launch");
  return IPB_OK;
}

// ---- non-maximum suppression ------------------------------------------------------
namespace {
ipb_status host_suppress(int type, size_t esize, const void* image, uint32_t W, uint32_t H, uint32_t radius,
                         void* out) {
  const size_t bytes = (size_t)W * H * esize;
  if ((!image && bytes) || (!out && bytes)) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  if (!bytes) return IPB_OK;  // empty image: empty output
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  if ((st = ensure(c, c->img, bytes)) || (st = ensure(c, c->out, bytes)) ||
      (st = ensure(c, c->scratch, suppress_scratch_bytes(type, W, H))))
    return st;
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(cudaMemcpyAsync(c->img.p, image, bytes, cudaMemcpyHostToDevice, c->stream), "copy image");
  IPB_CUDA(launch_suppress(type, c->img.p, W, H, radius, c->out.p, c->scratch.p, c->stream),
           "suppress_non_maximum launch");
  IPB_CUDA(cudaMemcpyAsync(out, c->out.p, bytes, cudaMemcpyDeviceToHost, c->stream), "copy output");
  return finish_sync(c, c->stream);
}

ipb_status device_suppress(int type, const void* d_image, uint32_t W, uint32_t H, uint32_t radius, void* d_out,
                           void* stream) {
  if (((size_t)W * H) && (!d_image || !d_out)) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  if (!((size_t)W * H)) return IPB_OK;
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  if ((st = ensure(c, c->scratch, suppress_scratch_bytes(type, W, H)))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  IPB_CUDA(cudaStreamWaitEvent(s, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(launch_suppress(type, d_image, W, H, radius, d_out, c->scratch.p, s),
           "suppress_non_maximum launch");
  IPB_CUDA(cudaEventRecord(c->last, s), "cudaEventRecord");
  return IPB_OK;
}
}  // namespace

#define IPB_DEFINE_SUPPRESS(T, S, CODE)                                                                  \
  IPB_API ipb_status ipb_suppress_non_maximum_##S(const T* image, uint32_t W, uint32_t H, uint32_t radius, \
                                                  T* out) {                                             \
    return host_suppress(CODE, sizeof(T), image, W, H, radius, out);                                     \
  }                                                                                                     \
  IPB_API ipb_status ipb_suppress_non_maximum_##S##_device(const T* d_image, uint32_t W, uint32_t H,      \
                                                           uint32_t radius, T* d_out, void* stream) {   \
    return device_suppress(CODE, d_image, W, H, radius, d_out, stream);                                  \
  }
IPB_DEFINE_SUPPRESS(uint8_t, u8, IPB_ELEM_U8)
IPB_DEFINE_SUPPRESS(uint16_t, u16, IPB_ELEM_U16)
IPB_DEFINE_SUPPRESS(uint32_t, u32, IPB_ELEM_U32)
IPB_DEFINE_SUPPRESS(uint64_t, u64, IPB_ELEM_U64)
IPB_DEFINE_SUPPRESS(int8_t, i8, IPB_ELEM_I8)
IPB_DEFINE_SUPPRESS(int16_t, i16, IPB_ELEM_I16)
IPB_DEFINE_SUPPRESS(int32_t, i32, IPB_ELEM_I32)
IPB_DEFINE_SUPPRESS(int64_t, i64, IPB_ELEM_I64)
IPB_DEFINE_SUPPRESS(float, f32, IPB_ELEM_F32)
#undef IPB_DEFINE_SUPPRESS

IPB_API ipb_status ipb_local_maxima(const uint32_t* xs, const uint32_t* ys, const float* scores, uint32_t n,
                                    uint32_t radius, uint32_t* out_indices, uint32_t* out_count) {
  if (!out_count || (n && (!xs || !ys || !scores || !out_indices)))
    return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  *out_count = 0;
  if (n == 0) return IPB_OK;
  uint32_t max_y = 0;  // sizes the row table; the kernels find the rows themselves
  for (uint32_t i = 0; i < n; ++i) max_y = ys[i] > max_y ? ys[i] : max_y;
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  const size_t nb = (size_t)n * 4;
  const size_t sb = local_maxima_scratch_bytes(n, max_y);
  if ((st = ensure(c, c->img, 4 * nb + 256)) || (st = ensure(c, c->scratch, sb))) return st;
  uint8_t* d = static_cast<uint8_t*>(c->img.p);
  uint32_t* d_xs = reinterpret_cast<uint32_t*>(d);
  uint32_t* d_ys = reinterpret_cast<uint32_t*>(d + nb);
  float* d_sc = reinterpret_cast<float*>(d + 2 * nb);
  uint32_t* d_out = reinterpret_cast<uint32_t*>(d + 3 * nb);
  uint32_t* d_count = reinterpret_cast<uint32_t*>(d + 4 * nb);
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(cudaMemcpyAsync(d_xs, xs, nb, cudaMemcpyHostToDevice, c->stream), "copy xs");
  IPB_CUDA(cudaMemcpyAsync(d_ys, ys, nb, cudaMemcpyHostToDevice, c->stream), "copy ys");
  IPB_CUDA(cudaMemcpyAsync(d_sc, scores, nb, cudaMemcpyHostToDevice, c->stream), "copy scores");
  IPB_CUDA(launch_local_maxima(d_xs, d_ys, d_sc, n, radius, max_y, c->scratch.p, sb, d_out, d_count, c->stream),
           "local_maxima launch");
  IPB_CUDA(cudaMemcpyAsync(out_count, d_count, 4, cudaMemcpyDeviceToHost, c->stream), "copy count");
  IPB_CUDA(cudaMemcpyAsync(out_indices, d_out, nb, cudaMemcpyDeviceToHost, c->stream), "copy indices");
  return finish_sync(c, c->stream);
}

// ---- filter_clamped -------------------------------------------------------------------
namespace {
size_t elem_size(int type) {
  switch (type) {
    case IPB_ELEM_U8: case IPB_ELEM_I8: return 1;
    case IPB_ELEM_U16: case IPB_ELEM_I16: return 2;
    case IPB_ELEM_U32: case IPB_ELEM_I32: case IPB_ELEM_F32: return 4;
    default: return 8;
  }
}

ipb_status check_filter_args(uint32_t channels, int ktype, uint32_t kw, uint32_t kh, int otype) {
  if (kw == 0 || kh == 0) return fail(IPB_ERR_INVALID_ARGUMENT, "width and height must be non-zero");
  if (channels != 1 && channels != 3 && channels != 4)
    return fail(IPB_ERR_INVALID_ARGUMENT, "channels must be 1 (Luma), 3 (Rgb) or 4 (Rgba)");
  if (!filter_types_supported(ktype, otype))
    return fail(IPB_ERR_INVALID_ARGUMENT,
                "no Clamp from this kernel type to this output type (f32 kernels: u8, u16, f32; i32 kernels: u8, "
                "u16, i16, i32)");
  return IPB_OK;
}
}  // namespace

IPB_API ipb_status ipb_filter_clamped(const uint8_t* image, uint32_t W, uint32_t H, uint32_t channels,
                                      const void* kernel, int kernel_type, uint32_t kw, uint32_t kh, int out_type,
                                      void* out) {
  ipb_status st = check_filter_args(channels, kernel_type, kw, kh, out_type);
  if (st) return st;
  const size_t ib = (size_t)W * H * channels, kb = (size_t)kw * kh * 4, ob = ib * elem_size(out_type);
  if (!kernel || ((!image || !out) && ib)) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  if (!ib) return IPB_OK;
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  if ((st = ensure(c, c->img, ib)) || (st = ensure(c, c->tpl, kb)) || (st = ensure(c, c->out, ob))) return st;
  IPB_CUDA(cudaStreamWaitEvent(c->stream, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(cudaMemcpyAsync(c->img.p, image, ib, cudaMemcpyHostToDevice, c->stream), "copy image");
  IPB_CUDA(cudaMemcpyAsync(c->tpl.p, kernel, kb, cudaMemcpyHostToDevice, c->stream), "copy kernel");
  IPB_CUDA(launch_filter(static_cast<const uint8_t*>(c->img.p), W, H, channels, c->tpl.p, kernel_type, kw, kh,
                         out_type, c->out.p, c->stream),
           "filter launch");
  IPB_CUDA(cudaMemcpyAsync(out, c->out.p, ob, cudaMemcpyDeviceToHost, c->stream), "copy output");
  return finish_sync(c, c->stream);
}

IPB_API ipb_status ipb_filter_clamped_device(const uint8_t* d_image, uint32_t W, uint32_t H, uint32_t channels,
                                             const void* d_kernel, int kernel_type, uint32_t kw, uint32_t kh,
                                             int out_type, void* d_out, void* stream) {
  ipb_status st = check_filter_args(channels, kernel_type, kw, kh, out_type);
  if (st) return st;
  if (!d_kernel || ((!d_image || !d_out) && (size_t)W * H)) return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  IPB_CUDA(launch_filter(d_image, W, H, channels, d_kernel, kernel_type, kw, kh, out_type, d_out,
                         static_cast<cudaStream_t>(stream)),
           "filter launch");
  return IPB_OK;
}

IPB_API ipb_status ipb_example_template_matching(const uint8_t* image, uint32_t W, uint32_t H, uint32_t tx,
                                                 uint32_t ty, uint32_t tw, uint32_t th, uint8_t* template_out,
                                                 uint8_t* image_rgb, uint8_t* sse_rgb, uint8_t* sse_norm_rgb) {
  // copy_sub_image's assertion (examples/template_matching.rs:79-82), in u64
  // so that no sum wraps
  if (!((uint64_t)tx + tw < W && (uint64_t)ty + th < H)) return fail(IPB_ERR_INVALID_ARGUMENT, "invalid sub-image");
  if (!tw || !th)
    return fail(IPB_ERR_INVALID_ARGUMENT,
                "an empty template's score map does not fit the padded canvas (the reference's copy_from "
                "fails with a dimension mismatch)");
  if (!image || !template_out || !image_rgb || !sse_rgb || !sse_norm_rgb)
    return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  ipb_status st;
  if ((st = get_ctx(&c))) return st;
  const size_t ib = (size_t)W * H, tb = (size_t)tw * th, rb = 3 * ib;
  const uint32_t Wo = W - tw + 1, Ho = H - th + 1;
  const size_t ob = (size_t)Wo * Ho * sizeof(float);
  if ((st = ensure(c, c->img, ib)) || (st = ensure(c, c->tpl, tb)) || (st = ensure(c, c->out, ob)) ||
      (st = ensure(c, c->rgb, rb)) || (st = ensure(c, c->keys, 2 * sizeof(uint32_t))))
    return st;
  cudaStream_t s = c->stream;
  const uint8_t* d_img = static_cast<const uint8_t*>(c->img.p);
  uint8_t* d_tpl = static_cast<uint8_t*>(c->tpl.p);
  uint8_t* d_rgb = static_cast<uint8_t*>(c->rgb.p);
  uint32_t* d_keys = static_cast<uint32_t*>(c->keys.p);
  // roi = Rect::at(tx as i32, ty as i32).of_size(tw, th): right/bottom inclusive
  const int32_t left = (int32_t)tx, top = (int32_t)ty;
  const int32_t right = left + (int32_t)tw - 1, bottom = top + (int32_t)th - 1;
  IPB_CUDA(cudaStreamWaitEvent(s, c->last, 0), "cudaStreamWaitEvent");
  IPB_CUDA(cudaMemcpyAsync(c->img.p, image, ib, cudaMemcpyHostToDevice, s), "copy image");
  IPB_CUDA(launch_crop(d_img, W, tx, ty, tw, th, d_tpl, s), "copy_sub_image");
  IPB_CUDA(cudaMemcpyAsync(template_out, d_tpl, tb, cudaMemcpyDeviceToHost, s), "copy template");
  IPB_CUDA(launch_render(d_img, nullptr, 0, 0, 0, 0, nullptr, W, H, left, top, right, bottom, d_rgb, s),
           "draw_green_rect");
  IPB_CUDA(cudaMemcpyAsync(image_rgb, d_rgb, rb, cudaMemcpyDeviceToHost, s), "copy image with roi");
  const int methods[2] = {IPB_SUM_OF_SQUARED_ERRORS, IPB_SUM_OF_SQUARED_ERRORS_NORMALIZED};
  uint8_t* outs[2] = {sse_rgb, sse_norm_rgb};
  for (int k = 0; k < 2; ++k) {
    MatchArgs a{d_img, W, H, d_tpl, tw, th, nullptr, false, methods[k], g_precision.load(),
                static_cast<float*>(c->out.p), s};
    if ((st = run_match(c, a))) return st;
    IPB_CUDA(launch_map_range(static_cast<const float*>(c->out.p), (size_t)Wo * Ho, d_keys, s), "score range");
    IPB_CUDA(launch_render(nullptr, static_cast<const float*>(c->out.p), Wo, Ho, tw / 2, th / 2, d_keys, W, H,
                           left, top, right, bottom, d_rgb, s),
             "rescale, pad and draw");
    IPB_CUDA(cudaMemcpyAsync(outs[k], d_rgb, rb, cudaMemcpyDeviceToHost, s), "copy result");
  }
  return finish_sync(c, s);
}

IPB_API ipb_status ipb_match_template_device(const uint8_t* d_image, uint32_t W, uint32_t H,
                                             const uint8_t* d_tpl, uint32_t w, uint32_t h,
                                             const uint8_t* d_mask, uint32_t mw, uint32_t mh,
                                             int mask_is_binary, int method, int precision, float* d_out,
                                             void* stream) {
  ipb_status st = check_match(W, H, w, h, d_mask != nullptr, mw, mh, method);
  if (st) return st;
  if (precision < 0 || precision > 2) return fail(IPB_ERR_INVALID_ARGUMENT, "unknown precision");
  if ((!d_image && (size_t)W * H) || (!d_tpl && (size_t)w * h) || !d_out)
    return fail(IPB_ERR_INVALID_ARGUMENT, "null buffer");
  Context* c = nullptr;
  if ((st = get_ctx(&c))) return st;
  MatchArgs a{d_image, W, H, d_tpl, w, h, d_mask, d_mask && mask_is_binary != 0, method, precision, d_out,
              static_cast<cudaStream_t>(stream)};
  return run_match(c, a);
}

#define IPB_DEFINE_FIND_EXTREMES(T, S)                                                            \
  IPB_API ipb_status ipb_find_extremes_##S(const T* image, uint32_t width, uint32_t height,        \
                                           ipb_extremes_##S* out) {                                \
    return extremes_host<T, ipb_extremes_##S>(image, width, height, out);                         \
  }                                                                                                \
  IPB_API ipb_status ipb_find_extremes_##S##_device(const T* d_image, uint32_t width,             \
                                                    uint32_t height, ipb_extremes_##S* out,        \
                                                    void* stream) {                                \
    return extremes_device<T, ipb_extremes_##S>(d_image, width, height, out, stream);             \
  }

IPB_DEFINE_FIND_EXTREMES(uint8_t, u8)
IPB_DEFINE_FIND_EXTREMES(uint16_t, u16)
IPB_DEFINE_FIND_EXTREMES(uint32_t, u32)
IPB_DEFINE_FIND_EXTREMES(uint64_t, u64)
IPB_DEFINE_FIND_EXTREMES(int8_t, i8)
IPB_DEFINE_FIND_EXTREMES(int16_t, i16)
IPB_DEFINE_FIND_EXTREMES(int32_t, i32)
IPB_DEFINE_FIND_EXTREMES(int64_t, i64)
IPB_DEFINE_FIND_EXTREMES(float, f32)
IPB_DEFINE_FIND_EXTREMES(double, f64)
