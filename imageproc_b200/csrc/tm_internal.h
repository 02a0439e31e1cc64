// tm_internal.h -- launchers shared between the kernel files and the C ABI.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>
#include <mutex>
#include <cuda_runtime.h>

namespace ipb {

// ---- per-device one-time set-up ------------------------------------------------
// A kernel's dynamic shared-memory limit (cudaFuncSetAttribute) belongs to the
// current device's context, not to the process: a process that uses two GPUs
// must set it on each. run(f) calls f() the first time it is reached with a
// given device current and returns cudaSuccess afterwards for that device; a
// failing f is tried again on the next call. Safe to call from many threads.
class PerDeviceOnce {
 public:
  template <typename F>
  cudaError_t run(F&& f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return f();  // beyond the bitmask: set every time
    const uint64_t bit = 1ull << dev;
    if (done_.load(std::memory_order_acquire) & bit) return cudaSuccess;
    std::lock_guard<std::mutex> g(mu_);
    if (done_.load(std::memory_order_relaxed) & bit) return cudaSuccess;
    e = f();
    if (e == cudaSuccess) done_.fetch_or(bit, std::memory_order_release);
    return e;
  }

 private:
  std::atomic<uint64_t> done_{0};
  std::mutex mu_;
};

// Streaming multiprocessors of the current device (cached per device).
int device_sm_count();

// Budget, in nanoseconds, of the bounded waits inside each tile of the
// tensor-core kernels (default 2 s). A wait that runs out stops the kernel's
// pipeline and reports IPB_ERR_TIMEOUT; the final wait for in-flight
// tensor-core work before tensor memory is freed always keeps the default.
// Lowered only by the test entry point ipb_debug_set_pipeline_wait_ns.
constexpr unsigned long long kDefaultWaitNs = 2000000000ull;
unsigned long long pipeline_wait_ns();
// Failure-detection test hook: when set, the MMA warp of every tensor-core
// kernel launched afterwards first waits on an mbarrier that nothing arrives
// at, so that bounded wait runs out (ipb_debug_stall_pipelines).
bool pipeline_stall();

// ---- tracing ---------------------------------------------------------------
// Every kernel launch site reports itself; the C ABI exposes the running
// count (ipb_launch_count) and, when profiling is on, CUDA-event timings of
// the dominant kernel of each call (ipb_profile_collect).
enum KernelId : int {
  kKernelPrep = 0,
  kKernelIntegralRows,
  kKernelIntegralCols,
  kKernelExactCC,
  kKernelTemplateSumF32,
  kKernelReference,
  kKernelExtremes,
  kKernelUmma,
  kKernelMany,
  kKernelSuppress,
  kKernelFilter,
  kKernelExample,
  kKernelLearned,
  kKernelPropose,
  kKernelRows,
  kKernelWindowSq,
  kKernelCount
};
const char* kernel_name(int id);
void count_launch(int id);

// Event pair recorded around a call's dominant kernel (both null = off).
struct KernelTimer {
  cudaEvent_t begin = nullptr;
  cudaEvent_t end = nullptr;
  int kernel = -1;  // set by the launcher: which kernel was timed
  uint32_t launches = 1;  // launches inside the span (concurrent launches timed together)
};

// One (image, template[, mask]) matching problem, all pointers on the device.
struct MatchArgs {
  const uint8_t* img;
  uint32_t W, H;
  const uint8_t* tpl;
  uint32_t w, h;
  const uint8_t* mask;  // nullptr when unmasked
  bool mask_binary;     // every mask value is 0 or 1
  int method;
  int precision;
  float* out;           // (W-w+1) x (H-h+1)
  cudaStream_t stream;
  KernelTimer* timer = nullptr;
};

inline void timer_begin(KernelTimer* t, int kernel, cudaStream_t s) {
  if (t && t->begin) {
    t->kernel = kernel;
    cudaEventRecord(t->begin, s);
  }
}
inline void timer_end(KernelTimer* t, cudaStream_t s) {
  if (t && t->end) cudaEventRecord(t->end, s);
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Records `msg` as the calling thread's ipb_last_error_message and returns st.
int report_error(int st, const char* msg);

// ---- template preparation (tm_prep.cu) ----------------------------------
// Byte planes of the template-side operands, each h rows of `pitch` bytes,
// zero beyond w, followed by the u64 template constant TSS.
//   unmasked: plane 0 = T
//   binary mask: plane 0 = T*m, plane 1 = m
//   general mask: planes 0..2 = bytes of T*m^2, planes 3..4 = bytes of m^2
int template_plane_count(const MatchArgs& a);
size_t template_pitch(uint32_t w);
size_t prep_scratch_bytes(const MatchArgs& a);
cudaError_t launch_prep(const MatchArgs& a, uint8_t* planes, unsigned long long* tss);

// ---- u64 integral image of I^2 (tm_integral.cu) --------------------------
// Exclusive summed-area table, (H+1) x (W+1) u64, S[y][x] = sum over y'<y,
// x'<x, the layout of imageproc's integral_squared_image
// (src/integral_image.rs:11-22, :89).
size_t integral_bytes(uint32_t W, uint32_t H);
cudaError_t launch_integral_squared(const uint8_t* img, uint32_t W, uint32_t H,
                                    unsigned long long* sat, cudaStream_t s);
cudaError_t launch_integral(const uint8_t* img, uint32_t W, uint32_t H,
                            unsigned long long* sat, cudaStream_t s);

// ---- integral-image API (tm_sat.cu) -----------------------------------------
// (W+1) x (H+1) x channels table of u32 (bits = 32, wrapping) or u64 sums of
// F or F^2, channels 1, 3 or 4 interleaved (src/integral_image.rs:50, :89).
cudaError_t launch_sat(const uint8_t* img, uint32_t W, uint32_t H, uint32_t channels, bool squared, int bits,
                       void* sat, cudaStream_t s);

// ---- non-maximum suppression (tm_suppress.cu) -------------------------------
// suppress_non_maximum of a W x H image of element `type` (ipb_elem_type);
// scratch = suppress_scratch_bytes (each pixel's row-window winner: column and key).
size_t suppress_scratch_bytes(int type, uint32_t W, uint32_t H);
cudaError_t launch_suppress(int type, const void* img, uint32_t W, uint32_t H, uint32_t r, void* out, void* scratch,
                            cudaStream_t s);
size_t local_maxima_scratch_bytes(uint32_t n, uint32_t max_y);
// local_maxima of n device points (max_y = the largest y): writes the kept
// points' input indices in the reference's order to out and their number to
// *count (both device memory).
cudaError_t launch_local_maxima(const uint32_t* xs, const uint32_t* ys, const float* scores, uint32_t n,
                                uint32_t radius, uint32_t max_y, void* scratch, size_t scratch_bytes,
                                uint32_t* out, uint32_t* count, cudaStream_t s);

// ---- filter_clamped (tm_filter.cu) --------------------------------------------
// whether the reference has a Clamp from the kernel type to the output type
bool filter_types_supported(int ktype, int otype);
// filter_clamped of a W x H u8 image with `channels` interleaved channels by a
// kw x kh row-major kernel (device memory); out is W x H x channels of otype.
cudaError_t launch_filter(const uint8_t* img, uint32_t W, uint32_t H, uint32_t channels, const void* kern, int ktype,
                          uint32_t kw, uint32_t kh, int otype, void* out, cudaStream_t s);

// ---- the example workflow of examples/template_matching.rs (tm_example.cu) ---
cudaError_t launch_crop(const uint8_t* img, uint32_t W, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                        uint8_t* out, cudaStream_t s);
// keys[0..1] <- order keys of the map's min and max, NaN skipped
cudaError_t launch_map_range(const float* map, size_t n, uint32_t* keys, cudaStream_t s);
// W x H x 3 RGB: the gray image (gray != null) or the map rescaled to u8 over
// keys' range and placed at (px, py), with the rectangle outline in green
cudaError_t launch_render(const uint8_t* gray, const float* map, uint32_t Wo, uint32_t Ho, uint32_t px,
                          uint32_t py, const uint32_t* keys, uint32_t W, uint32_t H, int32_t left, int32_t top,
                          int32_t right, int32_t bottom, uint8_t* rgb, cudaStream_t s);

// ---- CUDA-core exact kernel (tm_exact_cc.cu) ------------------------------
size_t exact_cc_scratch_bytes(const MatchArgs& a);
cudaError_t launch_exact_cc(const MatchArgs& a, void* scratch);

// ---- tensor-core exact kernel (tm_umma.cu) ---------------------------------
// One launch, no scratch: the kernel prepares the template side itself. A
// bounded wait that runs out stores `tag` into *err_word (atomicMax), so the
// word (zeroed once at allocation) tells whether a launch with that tag or a
// later one failed.
bool umma_supported(const MatchArgs& a);
cudaError_t launch_umma(const MatchArgs& a, unsigned int* err_word, unsigned int tag);

// ---- tensor-core exact kernel with the image row as the A operand (tm_shift.cu)
// Unmasked exact matches of images whose width is a multiple of 16 (rows
// 16-byte aligned); scratch = shift_scratch_bytes (the window sums of I^2,
// none for CrossCorrelation). ext: fused find_extremes keys {min, max} (armed
// by the caller) or null.
bool shift_supported(const MatchArgs& a);
// shift_supported and chosen by the kernel path setting (ipb_set_path)
bool shift_preferred(const MatchArgs& a);
size_t shift_scratch_bytes(const MatchArgs& a);
cudaError_t launch_shift(const MatchArgs& a, void* scratch, unsigned long long* ext, unsigned int* err_word,
                         unsigned int tag);
// Up to 8 problems with one template (same pointer and size) in one launch,
// each with its own extremes keys (ext[i], or ext null); problems on one image
// share its window sums. scratch = shift_multi_scratch_bytes.
constexpr uint32_t kShiftMaxProblems = 8;
size_t shift_multi_scratch_bytes(const MatchArgs* a, uint32_t n);
cudaError_t launch_shift_multi(const MatchArgs* a, unsigned long long* const* ext, uint32_t n, void* scratch,
                               unsigned int* err_word, unsigned int tag, cudaStream_t stream, KernelTimer* timer);

// One problem of a tensor-core launch (device-side descriptor).
struct UmmaProblem {
  const uint8_t* img;
  const uint8_t* tpl;
  const uint8_t* mask;       // binary mask or null
  float* out;
  unsigned long long* ext;   // fused find_extremes keys {min, max} or null
  uint32_t W, H, w, h;
  uint32_t Wo, Ho, tiles_x, tile_begin;  // tile_begin: first global tile of the problem
  uint32_t kmma, zrows, rows_max, load_mode;
  int method, precision;
  // Problems on one image with one template size (and one mask buffer) may
  // form a set that the kernel computes tile by tile together, sharing the
  // staged image rows and the A operand built from them (each member keeps
  // its own template side, X accumulator, MMAs and epilogue; a masked set's
  // Y = sum I^2 m, which depends on the image and the mask alone, is
  // computed once for all members). On a set's first problem: the number of
  // members (1 for a problem alone); 0 on the others, which follow it in the
  // problem list and carry its tile_begin. Tiles are counted per set.
  uint32_t set_n;
};

constexpr uint32_t kInlineProblems = 8;  // problems passed in the kernel parameters
constexpr uint32_t kMaxSet = 4;          // problems per set

struct UmmaLaunch {
  UmmaProblem inl[kInlineProblems];
  const UmmaProblem* probs;  // device array when nprobs > kInlineProblems
  uint32_t nprobs, tiles;
  uint32_t NT, rps, imgp, plane_bytes, nbuf;
  uint32_t z_off, img_off, rs_off;
  uint32_t set_max;  // largest set: accumulators and template buffers reserved per member
  unsigned int* err;
  unsigned int tag;
  // budget of the pipeline's bounded waits, per tile (pipeline_wait_ns())
  unsigned long long wait_ns;
  uint32_t stall;  // pipeline_stall() at launch
  // {next tile counter, CTAs finished}, both zero at launch: tiles after the
  // first wave are claimed from it; the last CTA out zeroes it again.
  // Null: a fixed grid stride.
  unsigned int* sched;
};

// Launch-wide plan of a group of problems sharing (tensor-memory row width,
// masked): tile height, pipeline depth and shared-memory carve.
struct UmmaPlan {
  uint32_t ks;
  bool masked;
  uint32_t NT, rps, imgp, plane_bytes, nbuf, z_off, img_off, rs_off, smem;
  uint32_t set_max;  // problems per set the plan holds (1..kMaxSet)
};

uint32_t umma_group_key(const MatchArgs& a);  // natural row width * 2 + masked
// Natural tensor-memory row width (8..64) of templates w pixels wide.
uint32_t umma_row_width(uint32_t w);
// Sets every tensor-core kernel's shared-memory limit (outside stream capture).
cudaError_t umma_prepare_kernels();
// Plan of a batch group (launches of many tiles): row width ks (8..64, a
// power of two; 32 at most with a mask), sets of up to `set` problems
// (1..kMaxSet) and the tile height nt, or the tallest tiles that fit when nt
// is 0. False when no plan fits.
bool umma_plan_for(uint32_t ks, bool masked, uint32_t hmax, UmmaPlan& pl, uint32_t nt = 0, uint32_t set = 1);
// The tile heights a batch group with sets of up to `set` problems can use,
// tallest first; returns the count.
uint32_t umma_tile_heights(bool masked, uint32_t set, uint32_t out[2]);
// Problems of a launch that share an image and a template size (and the mask
// kind): the size of the largest such class, at most kMaxSet.
uint32_t umma_largest_set(const std::vector<UmmaProblem>& probs);
// Reorders a launch's problems so that each class of the above follows
// itself, cuts the classes into sets of at most pl.set_max problems and
// numbers the sets' tiles from 0; returns the launch's tile count.
uint32_t umma_make_sets(std::vector<UmmaProblem>& probs, const UmmaPlan& pl);
UmmaProblem umma_problem(const MatchArgs& a, const UmmaPlan& pl, uint32_t tile_begin,
                         unsigned long long* ext_keys);
uint32_t umma_problem_tiles(const UmmaProblem& q, const UmmaPlan& pl);
// Fills the plan fields of L and launches (L.inl / L.probs, nprobs, tiles,
// err, tag set by the caller).
cudaError_t launch_umma_batch(const UmmaPlan& pl, UmmaLaunch& L, cudaStream_t stream, KernelTimer* timer);
// find_extremes keys (2 per template, armed by the caller) of n <= 8
// unmasked templates of one shape against one image, in one tensor-core
// launch without score maps.
cudaError_t launch_umma_extremes(const uint8_t* img, uint32_t W, uint32_t H, const uint8_t* const* tpls,
                                 uint32_t n, uint32_t w, uint32_t h, int method, int precision,
                                 unsigned long long* keys, unsigned int* err_word, unsigned int tag,
                                 cudaStream_t stream);
cudaError_t launch_extremes_keys_init(unsigned long long* keys, uint32_t n, cudaStream_t s);
// The finish kernel writes the records and re-arms the keys for the next launch.
cudaError_t launch_extremes_keys_finish(unsigned long long* keys, const uint32_t* widths,
                                        ipb_extremes_f32* const* outs, uint32_t n, cudaStream_t s);

// ---- many templates of one size against one image (tm_many.cu) ------------
bool many_supported(uint32_t w, uint32_t h, uint32_t n, int precision);
cudaError_t launch_many(const uint8_t* img, uint32_t W, uint32_t H, const uint8_t* tpl, uint32_t w, uint32_t h,
                        uint32_t n, int method, int precision, float* out, unsigned long long* ext_keys,
                        unsigned int* err, unsigned int tag, cudaStream_t stream, KernelTimer* timer);
cudaError_t launch_many_keys_init(unsigned long long* keys, uint32_t n, cudaStream_t s);
cudaError_t launch_many_keys_finish(const unsigned long long* keys, uint32_t Wo, ipb_extremes_f32* out, uint32_t n,
                                    cudaStream_t s);

// ---- reference-order f32 kernel (tm_reference.cu) -------------------------
size_t reference_scratch_bytes(const MatchArgs& a);
cudaError_t launch_reference(const MatchArgs& a, void* scratch);

// ---- find_extremes (tm_extremes.cu) ----------------------------------------
// Result record written to device memory by the reduction.
template <typename T>
struct ExtremesResult {
  T max_value;
  T min_value;
  unsigned long long max_index;
  unsigned long long min_index;
};
size_t extremes_scratch_bytes();
template <typename T>
cudaError_t launch_find_extremes(const T* d, unsigned long long n, void* scratch,
                                 ExtremesResult<T>* d_result, cudaStream_t s);
// ExtremesResult<float> of a map of the given width -> ipb_extremes_f32 (device)
cudaError_t launch_extremes_to_struct(const ExtremesResult<float>* r, uint32_t width, ipb_extremes_f32* out,
                                      cudaStream_t s);

// Validation shared by the single and batched entry points: the reference's
// assertions in its order; returns the status and sets the thread's message.
int check_match_args(uint32_t W, uint32_t H, uint32_t w, uint32_t h, bool masked, uint32_t mw, uint32_t mh,
                     int method);
void count_launches(unsigned long long n);
bool profiling_enabled();
KernelTimer* acquire_kernel_timer();
void note_kernel_timed(KernelTimer* t, double macs, double bytes);
int kernel_path();  // 0 auto, 1 CUDA cores, 2 tensor cores, 3 row-operand kernel

}  // namespace ipb
