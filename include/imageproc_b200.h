/*
 * imageproc_b200.h -- C ABI of the B200 (sm_100a) template-matching library.
 *
 * Drop-in boundary for imageproc's template-matching module
 * (imageproc 0.27.0, src/template_matching.rs). Every entry point below names
 * the reference item it replaces. Plain pointers and sizes only; every
 * function returns an ipb_status (0 = success) and, on failure, leaves a
 * message for ipb_last_error_message().
 *
 * Images are the reference's `Image<P>` layout (src/definitions.rs:14):
 * row-major, stride == width, no padding. Outputs of the match functions are
 * (width - template_width + 1) x (height - template_height + 1) f32 score maps
 * (src/template_matching.rs:420-424).
 *
 * Host-pointer entry points copy their inputs to the current CUDA device,
 * run there and copy the result back before returning (synchronous, like the
 * reference's functions). `_device` entry points take device pointers and a
 * cudaStream_t (passed as void*, NULL = legacy default stream) and only
 * enqueue work; results are ready when the stream is.
 *
 * There is no CPU fallback: without a usable sm_100 device every compute
 * entry point fails with IPB_ERR_CUDA or IPB_ERR_NO_DEVICE. Argument checks
 * run on the host before any device work, in the reference's order.
 */
#ifndef IMAGEPROC_B200_H
#define IMAGEPROC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
typedef enum ipb_status {
    IPB_OK = 0,
    /* "image width must be greater than or equal to template width"
     * (src/template_matching.rs:395-398) */
    IPB_ERR_TEMPLATE_WIDTH = 1,
    /* "image height must be greater than or equal to template height"
     * (src/template_matching.rs:399-402) */
    IPB_ERR_TEMPLATE_HEIGHT = 2,
    /* "the template and mask must be the same size"
     * (src/template_matching.rs:433-437) */
    IPB_ERR_MASK_SIZE = 3,
    /* "image must be non-empty" (src/template_matching.rs:483-486) */
    IPB_ERR_EMPTY_IMAGE = 4,
    IPB_ERR_INVALID_ARGUMENT = 5,
    IPB_ERR_CUDA = 6,
    IPB_ERR_NO_DEVICE = 7,
    IPB_ERR_OUT_OF_MEMORY = 8,
    IPB_ERR_TIMEOUT = 9
} ipb_status;

/* MatchTemplateMethod (src/template_matching.rs:8-64), same order. */
typedef enum ipb_method {
    IPB_SUM_OF_SQUARED_ERRORS = 0,
    IPB_SUM_OF_SQUARED_ERRORS_NORMALIZED = 1,
    IPB_CROSS_CORRELATION = 2,
    IPB_CROSS_CORRELATION_NORMALIZED = 3
} ipb_method;

/* Arithmetic of the score maps.
 *  EXACT_FP64 (default): exact integer window sums; SSE assembled as
 *    sum(I^2) - 2 sum(I*T) + sum(T^2); one f32 rounding of the integer score;
 *    normalised methods divide by sqrt(sum(I^2) * sum(T^2)) in FP64 and
 *    round once to f32.
 *  EXACT_F32: exact integer window sums, then the reference's own f32
 *    normalisation sequence (src/template_matching.rs:249-250).
 *  REFERENCE_F32: the reference's f32 accumulation order replicated
 *    (dy-outer, dx-inner sequential f32 sums, src/template_matching.rs:
 *    219-386), bit-identical to the reference on every input. */
typedef enum ipb_precision {
    IPB_PRECISION_EXACT_FP64 = 0,
    IPB_PRECISION_EXACT_F32 = 1,
    IPB_PRECISION_REFERENCE_F32 = 2
} ipb_precision;

/* Element types of arrays passed to the non-matching entry points
 * (suppression, filters): additive, no reference counterpart. */
typedef enum ipb_elem_type {
    IPB_ELEM_U8 = 0,
    IPB_ELEM_U16 = 1,
    IPB_ELEM_U32 = 2,
    IPB_ELEM_U64 = 3,
    IPB_ELEM_I8 = 4,
    IPB_ELEM_I16 = 5,
    IPB_ELEM_I32 = 6,
    IPB_ELEM_I64 = 7,
    IPB_ELEM_F32 = 8
} ipb_elem_type;

/* Accumulator (kernel element) type of filter_clamped. */
typedef enum ipb_kernel_type {
    IPB_KERNEL_TYPE_F32 = 0,
    IPB_KERNEL_TYPE_I32 = 1
} ipb_kernel_type;

/* Message of the last failure on the calling thread ("" if none). */
const char *ipb_last_error_message(void);

/* Library version string. */
const char *ipb_version(void);

/* Page-locked host memory from a process-wide cache (additive API; no
 * reference counterpart). Blocks freed with ipb_host_free are kept for reuse
 * (up to 1 GiB in total), so a caller that allocates a score map per call
 * gets memory that the device writes at the full link rate and that needs no
 * first-touch page faults. Returns NULL when no CUDA device is usable; the
 * entry points accept ordinary host memory as well. */
void *ipb_host_alloc(size_t bytes);
void ipb_host_free(void *ptr);
/* Return every cached (freed, unused) block to the driver; blocks still in
 * use are not affected. */
void ipb_host_cache_release(void);

/* Process-wide precision used by the reference-shaped entry points (the
 * ones without a precision argument). Default IPB_PRECISION_EXACT_FP64, or
 * the value of the environment variable IPB_PRECISION (0, 1, 2 or
 * exact_fp64 / exact_f32 / reference_f32) at load time. */
ipb_status ipb_set_precision(int precision);
int ipb_get_precision(void);

/* Kernel family of the exact precisions (no counterpart in the reference):
 * 0 = automatic (tcgen05 tensor cores where the template shape allows, else
 * CUDA cores), 1 = CUDA cores only, 2 = tensor cores wherever supported,
 * 3 = the tensor-core kernel that reads image rows as its A operand
 * (unmasked, image width a multiple of 16) wherever it applies, else as 0.
 * Results are identical; the switch exists for testing and measurement.
 * Initial value from the environment variable IPB_PATH (0/1/2 or
 * auto/cuda_core/tensor). */
ipb_status ipb_set_path(int path);
int ipb_get_path(void);

/* Failure-detection test hook (no counterpart in the reference): the budget,
 * in nanoseconds, of the bounded waits inside each tile of the tensor-core
 * kernels; 0 restores the default of 2 s. A wait that runs out stops the
 * kernel's pipeline, lets its tensor-core work drain (that last wait keeps the
 * 2 s budget), frees its tensor memory and makes the call report
 * IPB_ERR_TIMEOUT; the context stays usable. Takes effect for launches
 * planned after the call (batch plans keep the budget they were made with).
 * Tests set a budget far below one tile's time to make a wait run out without
 * faulting or hanging the GPU. */
void ipb_debug_set_pipeline_wait_ns(uint64_t ns);
/* Failure-detection test hook (no counterpart in the reference): while
 * enabled, the MMA-issuing warp of every tensor-core kernel launched
 * afterwards first waits on a barrier that nothing arrives at, so its bounded
 * wait runs out and the call reports IPB_ERR_TIMEOUT; pair it with a small
 * budget from ipb_debug_set_pipeline_wait_ns to keep the test short. Nothing
 * faults or spins without a limit. */
void ipb_debug_stall_pipelines(int enable);

/* ---- tracing -------------------------------------------------------------
 * No counterpart in the reference (which has no instrumentation); used by the
 * benchmark and the profiling notes. */

/* Number of kernels this library has launched in the process so far. */
uint64_t ipb_launch_count(void);

/* When enabled, each matching call records CUDA events around its dominant
 * kernel on the call's stream. */
ipb_status ipb_profile_enable(int enable);

typedef struct ipb_kernel_stats {
    const char *name;         /* kernel family */
    uint64_t launches;        /* timed launches */
    double total_ms;          /* summed event time of those launches */
    double algorithmic_macs;  /* summed (W-w+1)(H-h+1)*w*h */
    double algorithmic_bytes; /* summed image + template (+mask) + f32 output */
} ipb_kernel_stats;

/* Waits for the recorded events, writes up to max_entries per-kernel records
 * (those with at least one timed launch), resets the counters and returns
 * the number of records available. */
int ipb_profile_collect(ipb_kernel_stats *out, int max_entries);

/* ---- match_template ------------------------------------------------------ */

/* match_template (src/template_matching.rs:78-92). */
ipb_status ipb_match_template(const uint8_t *image, uint32_t image_width,
                              uint32_t image_height, const uint8_t *templ,
                              uint32_t template_width,
                              uint32_t template_height, int method,
                              float *out);

/* match_template_parallel (src/template_matching.rs:96-110). The reference
 * computes the same values as match_template with rows on rayon threads;
 * here both run the same device path, so results are identical. */
ipb_status ipb_match_template_parallel(const uint8_t *image,
                                       uint32_t image_width,
                                       uint32_t image_height,
                                       const uint8_t *templ,
                                       uint32_t template_width,
                                       uint32_t template_height, int method,
                                       float *out);

/* match_template_with_mask (src/template_matching.rs:125-140). The mask is a
 * GrayImage of its own size; its size must equal the template's. Mask values
 * are arbitrary u8 weights, as in the reference. */
ipb_status ipb_match_template_with_mask(
    const uint8_t *image, uint32_t image_width, uint32_t image_height,
    const uint8_t *templ, uint32_t template_width, uint32_t template_height,
    int method, const uint8_t *mask, uint32_t mask_width,
    uint32_t mask_height, float *out);

/* match_template_with_mask_parallel (src/template_matching.rs:144-163). */
ipb_status ipb_match_template_with_mask_parallel(
    const uint8_t *image, uint32_t image_width, uint32_t image_height,
    const uint8_t *templ, uint32_t template_width, uint32_t template_height,
    int method, const uint8_t *mask, uint32_t mask_width,
    uint32_t mask_height, float *out);

/* Device-resident form of the four functions above with an explicit
 * precision. mask may be NULL (unmasked); mask_is_binary != 0 asserts every
 * mask value is 0 or 1, which selects the cheaper binary-mask plan (a
 * non-binary mask under that flag gives wrong scores, so pass 0 when in
 * doubt). Replaces the same reference items as the host forms. */
ipb_status ipb_match_template_device(
    const uint8_t *d_image, uint32_t image_width, uint32_t image_height,
    const uint8_t *d_templ, uint32_t template_width, uint32_t template_height,
    const uint8_t *d_mask, uint32_t mask_width, uint32_t mask_height,
    int mask_is_binary, int method, int precision, float *d_out,
    void *stream);

/* ipb_match_template_device without any memory allocation. No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc (a plug-in
 * inside an application that owns the device-memory budget, a latency-critical
 * loop where cudaMalloc/cudaFree would stall or synchronise the device, code
 * that must not hit an out-of-memory failure after start-up). Same arguments
 * and the same scores as ipb_match_template_device; the caller still passes
 * inputs and outputs. It runs the CUDA-core kernels only (no tensor-core
 * path), so large templates can take several times longer than through
 * ipb_match_template_device. Its scratch memory is a fixed 16 MiB array inside the library,
 * which every GPU that loads the library holds until the process exits;
 * problems needing more (the u64 integral image of an unmasked SSE or
 * normalised match takes (W+1)(H+1)*8 bytes, so images up to about 2.09
 * megapixels) fail with IPB_ERR_INVALID_ARGUMENT and a message naming the
 * size. The first call on each device looks up the array's device address
 * (make it before any stream capture) and keeps it for the life of the
 * process, so a device reset (cudaDeviceReset) is not supported afterwards,
 * as for the rest of this library. All calls share the array: calls that
 * overlap on the GPU race on it and must be ordered by the caller. */
ipb_status ipb_match_template_device_noalloc(
    const uint8_t *d_image, uint32_t image_width, uint32_t image_height,
    const uint8_t *d_templ, uint32_t template_width, uint32_t template_height,
    const uint8_t *d_mask, uint32_t mask_width, uint32_t mask_height,
    int mask_is_binary, int method, int precision, float *d_out,
    void *stream);

/* ---- batches --------------------------------------------------------------
 * Many (image, template[, mask]) pairs of uneven sizes and methods in one
 * call: the reference's match_template / match_template_with_mask
 * (src/template_matching.rs:78, :125) applied per pair, optionally followed
 * by find_extremes (:479) of each score map. Additive API (the reference has
 * no batch form). Pairs are checked in order with the reference's assertions
 * before any work; the first failing pair's status is returned and its index
 * named in the message. Tensor-core pairs of equal tensor-memory row width
 * share one persistent launch each; find_extremes is fused into their
 * epilogue. */

typedef struct ipb_extremes_f32 ipb_extremes_f32;

typedef struct ipb_pair {
    const uint8_t *image; /* device */
    uint32_t image_width, image_height;
    const uint8_t *templ; /* device */
    uint32_t template_width, template_height;
    const uint8_t *mask; /* device, NULL = unmasked */
    uint32_t mask_width, mask_height;
    int mask_is_binary; /* every mask value is 0 or 1 */
    int method;
    float *out;                  /* device score map */
    ipb_extremes_f32 *extremes;  /* device record filled with find_extremes(out), or NULL */
} ipb_pair;

/* Enqueue the whole batch on `stream`. */
ipb_status ipb_match_template_batch_device(const ipb_pair *pairs, uint32_t n,
                                           int precision, void *stream);

/* A reusable batch: pairs checked, kernel paths chosen, tensor-core pairs
 * grouped into one launch per (row width, tile height, mask kind), device
 * descriptors uploaded and the launch sequence captured in a CUDA graph.
 * Autotuning (environment variable IPB_AUTOTUNE): unset, each group's row
 * width (its natural width or twice it) and tile height are timed on the
 * group's own pairs the first time a group of that class is planned, so plan
 * creation may run the pairs and write their outputs; IPB_AUTOTUNE=1 also
 * times tensor cores against the CUDA-core kernel per template shape class;
 * IPB_AUTOTUNE=0 uses the cost model alone. Decisions are cached per process
 * and persisted in IPB_TUNING_FILE (default ~/.cache/imageproc_b200/
 * tuning.txt; an empty value keeps them in memory).
 * Pointers in `pairs` must stay valid for the plan's life; launching replays
 * the graph on `stream`. Tensor-core groups run side by side inside the graph
 * (a fork to the plan's own stream and a join back), so the launch is ordered
 * on `stream` like one kernel. A plan holds one set of outputs and tile
 * counters: launch it again only in stream order after the previous launch,
 * never on two streams at once. */
typedef struct ipb_batch_plan ipb_batch_plan;
ipb_status ipb_batch_plan_create(const ipb_pair *pairs, uint32_t n, int precision,
                                 ipb_batch_plan **plan);
ipb_status ipb_batch_plan_launch(ipb_batch_plan *plan, void *stream);
/* Kernels one launch of the plan runs, and how many pairs use tensor cores. */
ipb_status ipb_batch_plan_info(const ipb_batch_plan *plan, uint32_t *kernels,
                               uint32_t *tensor_pairs);
/* The plan's tensor-core launches, in launch order: up to `max` records and
 * their total count in *count. */
typedef struct ipb_batch_group {
    uint32_t row_width; /* tensor-memory row width (8..64 bytes per image row segment) */
    uint32_t tile_rows; /* output rows per tile */
    int masked;         /* binary-mask launch */
    uint32_t pairs;     /* pairs in the launch */
    uint32_t tiles;     /* tiles the launch's CTAs share */
    uint32_t set_size;  /* pairs on one image computed together per tile (1..4) */
} ipb_batch_group;
ipb_status ipb_batch_plan_groups(const ipb_batch_plan *plan, uint32_t max, ipb_batch_group *out,
                                 uint32_t *count);
/* Forget the process's tuning decisions; the next plan re-reads the tuning
 * file (IPB_TUNING_FILE as it is then). */
void ipb_batch_tuning_reset(void);
ipb_status ipb_batch_plan_destroy(ipb_batch_plan *plan);

/* The tensor-core tile plan that a template of w x h pixels (binary mask or
 * not) gets: in a launch of its own (batch = 0: one map, or one row band of a
 * host-buffer call) or in a batch-plan group (batch = 1). Host arithmetic
 * only, no device work. Replaces no reference function: it describes this
 * library's launches. IPB_ERR_INVALID_ARGUMENT when the tensor path does not
 * take the shape (such templates run on CUDA cores). */
typedef struct ipb_tensor_plan {
    uint32_t tile_rows;      /* output rows per tile (a tile is 128 columns wide) */
    uint32_t image_rows;     /* image rows a tile reads: tile_rows + h - 1 */
    uint32_t rows_per_stage; /* image rows per tensor-memory pipeline stage */
    uint32_t stages;         /* pipeline stages */
    uint32_t image_buffers;  /* 2: the next tile's rows load during this one */
    uint32_t tmem_columns;   /* accumulators + A stages, of the 512 per SM */
    uint32_t smem_bytes;     /* dynamic shared memory per CTA */
} ipb_tensor_plan;
ipb_status ipb_tensor_plan_for(uint32_t w, uint32_t h, int masked, int batch, ipb_tensor_plan *out);
/* The same view for a batch group whose pairs on one image (one template
 * size, one mask kind) are computed together in sets of problems_per_set
 * (1..4): a tile's staged image rows and the A operand built from them serve
 * every member, each with its own template side and accumulators
 * (tmem_columns counts every member's). Replaces no reference function;
 * IPB_ERR_INVALID_ARGUMENT when no such plan fits (the batch planner then
 * computes those pairs alone). */
ipb_status ipb_tensor_set_plan_for(uint32_t w, uint32_t h, int masked, uint32_t problems_per_set,
                                   ipb_tensor_plan *out);

/* ---- many templates against one image --------------------------------------
 * match_template (src/template_matching.rs:78-92) of n templates of one size
 * w x h against one image, unmasked, in one launch on the tensor cores
 * (additive API). d_templates holds the n w x h GrayImages back to back.
 * Scores are POSITION-MAJOR: the score of template t at (x, y) is
 * d_out[((size_t)y * (W - w + 1) + x) * n + t]. d_out may be NULL when only
 * d_extremes (n records, find_extremes of each template's map,
 * src/template_matching.rs:479-511) is wanted. Templates of 16..64 columns
 * and 1..64 rows, EXACT precisions; other shapes go through
 * ipb_match_template_batch_device. Enqueued on `stream`. */
ipb_status ipb_match_templates_device(const uint8_t *d_image, uint32_t image_width,
                                      uint32_t image_height, const uint8_t *d_templates,
                                      uint32_t template_width, uint32_t template_height,
                                      uint32_t n_templates, int method, int precision,
                                      float *d_out, ipb_extremes_f32 *d_extremes,
                                      void *stream);

/* ---- learned proposals -------------------------------------------------------
 * Additive API with no counterpart in the reference, which scores every
 * window. For many 48 x 48 templates against one large image, a small
 * convolutional network (bf16 weights, fp32 accumulation) proposes windows;
 * their scores are computed exactly, a lower bound on every other window
 * certifies the answer, and templates that cannot be certified (or whose
 * heatmap margin is low) are answered by the exhaustive kernel. The answer
 * is what match_template (src/template_matching.rs:78-92) followed by
 * find_extremes (:479-511) gives for SumOfSquaredErrors: the first minimum in
 * row-major order of the EXACT_FP64 score map.
 *
 * The network: 4 x 4 box downsample, five 3 x 3 convolutions of 32 channels
 * (ReLU after the first four), and a 2 x 2 x 32 embedding of each template
 * (the same layers applied to the template) correlated with the image's
 * features. Parameters are IPB_PROPOSAL_NET_PARAMS fp32 values:
 * W1 [32][1][3][3], b1 [32], then W2..W5 [32][32][3][3] each followed by its
 * bias [32]. */
#define IPB_PROPOSAL_NET_PARAMS 37312
typedef struct ipb_proposal_net ipb_proposal_net;

/* A network on the current device with the given parameters (host array). */
ipb_status ipb_proposal_net_create(const float *params, ipb_proposal_net **net);
ipb_status ipb_proposal_net_destroy(ipb_proposal_net *net);
/* The current parameters (host array of IPB_PROPOSAL_NET_PARAMS floats). */
ipb_status ipb_proposal_net_get_params(const ipb_proposal_net *net, float *params);

/* Training. A batch is n_scenes crops of scene_height x scene_width u8
 * (sides multiples of 4) and n_templates (<= 128) 48 x 48 templates, all on
 * the device, back to back. d_positives (device, int64, one per template)
 * holds each template's target heatmap position as a flat index into the
 * crops' downsampled positions: (crop * (scene_height / 4) + py) *
 * (scene_width / 4) + px, where (px, py) = the downsampled position of the
 * template's best window (from the exhaustive kernel) plus 5. The loss is the
 * softmax cross-entropy of each template's logits over all positions of all
 * crops. _gradients writes the loss and the gradients (host, same layout as
 * the parameters); _train_step takes one Adam step (beta 0.9, 0.999). */
ipb_status ipb_proposal_net_gradients(ipb_proposal_net *net, const uint8_t *d_scenes, uint32_t n_scenes,
                                      uint32_t scene_height, uint32_t scene_width,
                                      const uint8_t *d_templates, uint32_t n_templates,
                                      const int64_t *d_positives, float *h_loss, float *h_grads,
                                      void *stream);
ipb_status ipb_proposal_net_train_step(ipb_proposal_net *net, const uint8_t *d_scenes, uint32_t n_scenes,
                                       uint32_t scene_height, uint32_t scene_width,
                                       const uint8_t *d_templates, uint32_t n_templates,
                                       const int64_t *d_positives, float learning_rate, float *h_loss,
                                       void *stream);

/* The network's features of one image (device, sides non-zero multiples of 4):
 * d_out receives (height / 4) x 4 x (width / 4) units of 8 bf16 channels, unit
 * (y, c, x) at index (y * 4 + c) * (width / 4) + x holding channels 8c .. 8c + 7
 * of position (x, y). kernel 0 runs the 32-channel layers on tcgen05 (the
 * query path), 1 on mma.sync (the training path); both accumulate in fp32. */
ipb_status ipb_proposal_net_features(ipb_proposal_net *net, const uint8_t *d_image, uint32_t width,
                                     uint32_t height, int kernel, void *d_out, void *stream);

typedef struct ipb_propose_options {
    uint32_t top_k;    /* windows of 32 x 32 positions verified per template (1..16, default 16) */
    float min_margin;  /* heatmap confidence margin below which a template falls back (default 0.1) */
    int certify;       /* 1 (default): certify answers; 0: accept the verified windows' best */
} ipb_propose_options;

typedef struct ipb_proposal_result {
    float value;        /* the minimum SumOfSquaredErrors score */
    uint32_t x, y;      /* its first location in row-major order */
    float margin;       /* the heatmap's confidence margin */
    uint32_t path;      /* 0: proposals, verified and certified; 1: fallback (low margin);
                           2: fallback (not certified) */
    uint32_t uncertified; /* blocks of 4 x 4 positions the certificate could not exclude
                             outside the proposed windows (verified exactly when at most 16384) */
} ipb_proposal_result;

/* Answers n_templates SumOfSquaredErrors queries of 48 x 48 templates
 * (device, back to back) against one image (device; sides multiples of 32)
 * and writes one result per template to `results` (host). options may be
 * NULL (defaults). Synchronises `stream` before returning. */
ipb_status ipb_propose_and_match_device(const ipb_proposal_net *net, const uint8_t *d_image,
                                        uint32_t image_width, uint32_t image_height,
                                        const uint8_t *d_templates, uint32_t template_width,
                                        uint32_t template_height, uint32_t n_templates, int method,
                                        const ipb_propose_options *options, ipb_proposal_result *results,
                                        void *stream);

/* The same queries with the proposals given instead of the network's: k
 * (1..16) template origins per template in d_origins (device, n_templates x k,
 * y * (image_width - 47) + x), each the centre of a 32 x 32 window of
 * positions scored exactly, then the same certification and exhaustive
 * fallback (options: certify; top_k and min_margin are ignored, margins are
 * +inf). Used to compare proposal sources on equal terms. */
ipb_status ipb_match_proposals_device(const uint8_t *d_image, uint32_t image_width, uint32_t image_height,
                                      const uint8_t *d_templates, uint32_t template_width,
                                      uint32_t template_height, uint32_t n_templates, int method,
                                      const uint32_t *d_origins, uint32_t k,
                                      const ipb_propose_options *options, ipb_proposal_result *results,
                                      void *stream);

/* ---- find_extremes -------------------------------------------------------- */

/* Extremes<T> (src/template_matching.rs:463-475), field order kept. */
#define IPB_DECLARE_EXTREMES(T, S)                                            \
    typedef struct ipb_extremes_##S {                                         \
        T max_value;                                                          \
        T min_value;                                                          \
        uint32_t max_value_location_x, max_value_location_y;                  \
        uint32_t min_value_location_x, min_value_location_y;                  \
    } ipb_extremes_##S;

IPB_DECLARE_EXTREMES(uint8_t, u8)
IPB_DECLARE_EXTREMES(uint16_t, u16)
IPB_DECLARE_EXTREMES(uint32_t, u32)
IPB_DECLARE_EXTREMES(uint64_t, u64)
IPB_DECLARE_EXTREMES(int8_t, i8)
IPB_DECLARE_EXTREMES(int16_t, i16)
IPB_DECLARE_EXTREMES(int32_t, i32)
IPB_DECLARE_EXTREMES(int64_t, i64)
IPB_DECLARE_EXTREMES(float, f32)
IPB_DECLARE_EXTREMES(double, f64)

/* find_extremes<T> (src/template_matching.rs:479-511) for every Primitive
 * channel type (usize/isize map to the 64-bit forms). Ties resolve to the
 * first pixel in row-major order; a NaN at (0, 0) is returned for both
 * extremes, other NaNs are skipped, exactly like the reference's strict
 * comparisons. Empty images fail with IPB_ERR_EMPTY_IMAGE. */
#define IPB_DECLARE_FIND_EXTREMES(T, S)                                       \
    ipb_status ipb_find_extremes_##S(const T *image, uint32_t width,          \
                                     uint32_t height,                         \
                                     ipb_extremes_##S *out);                  \
    ipb_status ipb_find_extremes_##S##_device(const T *d_image,               \
                                              uint32_t width,                 \
                                              uint32_t height,                \
                                              ipb_extremes_##S *out,          \
                                              void *stream);

IPB_DECLARE_FIND_EXTREMES(uint8_t, u8)
IPB_DECLARE_FIND_EXTREMES(uint16_t, u16)
IPB_DECLARE_FIND_EXTREMES(uint32_t, u32)
IPB_DECLARE_FIND_EXTREMES(uint64_t, u64)
IPB_DECLARE_FIND_EXTREMES(int8_t, i8)
IPB_DECLARE_FIND_EXTREMES(int16_t, i16)
IPB_DECLARE_FIND_EXTREMES(int32_t, i32)
IPB_DECLARE_FIND_EXTREMES(int64_t, i64)
IPB_DECLARE_FIND_EXTREMES(float, f32)
IPB_DECLARE_FIND_EXTREMES(double, f64)

/* ---- integral images ---------------------------------------------------------
 * integral_image / integral_squared_image (src/integral_image.rs:50, :89,
 * implementation :98-153) of a u8 image with `channels` interleaved channels
 * (1 = Luma, 3 = Rgb, 4 = Rgba): a (width + 1) x (height + 1) table, row-major,
 * `channels` values per entry, entry (x, y) = sum of F(x', y') (or F(x', y')^2)
 * over x' < x, y' < y, so the top row and the left column are zero. The u32
 * forms wrap modulo 2^32 like the reference's u32 sums in a release build; the
 * u64 forms are exact. An empty image gives a table of zeros.
 * sum_image_pixels and variance (:250, :303) are O(1) lookups into these
 * tables and live in the C++ and Python mirrors. */
ipb_status ipb_integral_image_u32(const uint8_t *image, uint32_t width, uint32_t height,
                                  uint32_t channels, uint32_t *out);
ipb_status ipb_integral_squared_image_u32(const uint8_t *image, uint32_t width, uint32_t height,
                                          uint32_t channels, uint32_t *out);
ipb_status ipb_integral_image_u64(const uint8_t *image, uint32_t width, uint32_t height,
                                  uint32_t channels, uint64_t *out);
ipb_status ipb_integral_squared_image_u64(const uint8_t *image, uint32_t width, uint32_t height,
                                          uint32_t channels, uint64_t *out);
/* The same on device buffers, enqueued on `stream`; bits = 32 or 64. */
ipb_status ipb_integral_image_device(const uint8_t *d_image, uint32_t width, uint32_t height,
                                     uint32_t channels, int squared, int bits, void *d_out,
                                     void *stream);

/* ---- non-maximum suppression ---------------------------------------------------
 * suppress_non_maximum (src/suppress.rs:10-107) for the reference's integer
 * channel types (Primitive + Ord; usize/isize map to the 64-bit forms): `out`
 * (width x height, row-major) holds a pixel's value where it is the greatest
 * in the (2 * radius + 1)^2 window centred on it (clipped to the image) and
 * zero elsewhere; among equal values the lexicographically smaller (x, y)
 * wins. The f32 form is additive (f32 is not Ord in the reference), for score
 * maps: values compare in IEEE total order (-0 below +0, NaN above every
 * number). The device
 * forms are enqueued on `stream` and use the calling thread's scratch. */
#define IPB_DECLARE_SUPPRESS(T, S)                                                        \
    ipb_status ipb_suppress_non_maximum_##S(const T *image, uint32_t width, uint32_t height, \
                                            uint32_t radius, T *out);                    \
    ipb_status ipb_suppress_non_maximum_##S##_device(const T *d_image, uint32_t width,      \
                                                     uint32_t height, uint32_t radius,     \
                                                     T *d_out, void *stream);

IPB_DECLARE_SUPPRESS(uint8_t, u8)
IPB_DECLARE_SUPPRESS(uint16_t, u16)
IPB_DECLARE_SUPPRESS(uint32_t, u32)
IPB_DECLARE_SUPPRESS(uint64_t, u64)
IPB_DECLARE_SUPPRESS(int8_t, i8)
IPB_DECLARE_SUPPRESS(int16_t, i16)
IPB_DECLARE_SUPPRESS(int32_t, i32)
IPB_DECLARE_SUPPRESS(int64_t, i64)
IPB_DECLARE_SUPPRESS(float, f32)

/* local_maxima (src/suppress.rs:111-173) of n scored points (x, y, score):
 * writes to out_indices the input indices of the points the reference
 * returns, in its order (points sorted by (y, x), equal positions in input
 * order), and their number to *out_count. out_indices holds n entries. */
ipb_status ipb_local_maxima(const uint32_t *xs, const uint32_t *ys, const float *scores, uint32_t n,
                            uint32_t radius, uint32_t *out_indices, uint32_t *out_count);

/* ---- filters ---------------------------------------------------------------------
 * filter_clamped (src/filter/mod.rs:202-212, through filter :29-70): the 2-D
 * correlation of a u8 image with `channels` interleaved channels (1, 3, 4) by a
 * kernel_width x kernel_height row-major kernel of kernel_type (f32 or i32),
 * padded by continuity, accumulated per channel in the kernel's type in the
 * reference's order (rows of the kernel outer, columns inner; f32 rounds each
 * multiply and add; i32 wraps like a release build) and clamped to out_type by
 * the reference's Clamp (src/definitions.rs:114-190): f32 kernels to u8, u16
 * or f32, i32 kernels to u8, u16, i16 or i32. Output: width x height x
 * channels of out_type. A kernel with a zero side fails with the reference's
 * message "width and height must be non-zero" (src/kernel.rs:25). With 1 x n
 * and n x 1 kernels this is horizontal_filter / vertical_filter
 * (src/filter/mod.rs:232, :319). */
ipb_status ipb_filter_clamped(const uint8_t *image, uint32_t width, uint32_t height, uint32_t channels,
                              const void *kernel, int kernel_type, uint32_t kernel_width,
                              uint32_t kernel_height, int out_type, void *out);
/* The same on device buffers (the kernel too), enqueued on `stream`. */
ipb_status ipb_filter_clamped_device(const uint8_t *d_image, uint32_t width, uint32_t height,
                                     uint32_t channels, const void *d_kernel, int kernel_type,
                                     uint32_t kernel_width, uint32_t kernel_height, int out_type,
                                     void *d_out, void *stream);

/* ---- the example workflow ----------------------------------------------------------
 * What examples/template_matching.rs main (:136-190) computes after decoding
 * its input, as one device pipeline over a width x height Luma image:
 *   template_out  (tw x th)   copy_sub_image(image, tx, ty, tw, th) (:78-92),
 *                             which asserts tx + tw < width and ty + th < height
 *                             ("invalid sub-image");
 *   image_rgb     (W x H x 3) draw_green_rect(image, roi) (:94-98): the image
 *                             as RGB with the outline of roi = Rect::at(tx, ty)
 *                             .of_size(tw, th) in (0, 255, 0);
 *   sse_rgb, sse_norm_rgb     run_match_template (:100-134) for
 *                             SumOfSquaredErrors and its normalised form: the
 *                             score map (at the library's precision) rescaled
 *                             to u8 by convert_to_gray_image (:63-76), placed in
 *                             a W x H canvas at (tw/2, th/2), drawn with roi.
 * The example's `parallel` argument selects match_template_parallel, whose
 * scores are identical; it has no counterpart here. tw and th must be non-zero
 * (the reference fails placing an empty template's map: a dimension mismatch). */
ipb_status ipb_example_template_matching(const uint8_t *image, uint32_t width, uint32_t height, uint32_t tx,
                                         uint32_t ty, uint32_t tw, uint32_t th, uint8_t *template_out,
                                         uint8_t *image_rgb, uint8_t *sse_rgb, uint8_t *sse_norm_rgb);

#ifdef __cplusplus
}
#endif
#endif /* IMAGEPROC_B200_H */
