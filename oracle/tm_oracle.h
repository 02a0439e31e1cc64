/*
 * tm_oracle.h -- CPU oracle for imageproc's template-matching path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA path: only the
 * test-suite, the smoke check and the CPU-baseline leg of the benchmark call
 * it. No product code path links against it.
 *
 * Parity status: pinned. The reference (imageproc 0.27.0, Rust) cannot be
 * compiled here, so this restatement is pinned against every known-answer
 * test the reference holds for the path (src/template_matching.rs:518-833),
 * extracted as text into tests/golden/reference_unit_tests.json.
 *
 * Three arithmetic flavours:
 *   tmo_match_reference  the reference's own f32 op sequence, bit for bit
 *                        (src/template_matching.rs:219-386, walk :405-456);
 *   tmo_sums             exact u64 integer sums X = sum(I*U), Y = sum(I^2*V)
 *                        and the template constant TSS;
 *   tmo_match_exact      exact sums + FP64 normalisation (precision 0) or
 *                        exact sums + the reference's f32 normalisation
 *                        (precision 1).
 */
#ifndef TM_ORACLE_H
#define TM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TMO_SSE = 0,
    TMO_SSE_NORMALIZED = 1,
    TMO_CCORR = 2,
    TMO_CCORR_NORMALIZED = 3
};

enum { TMO_PRECISION_EXACT_FP64 = 0, TMO_PRECISION_EXACT_F32 = 1 };

/* Status codes mirror the library's (include/imageproc_b200.h). */
enum {
    TMO_OK = 0,
    TMO_ERR_TEMPLATE_WIDTH = 1,
    TMO_ERR_TEMPLATE_HEIGHT = 2,
    TMO_ERR_MASK_SIZE = 3,
    TMO_ERR_EMPTY_IMAGE = 4,
    TMO_ERR_INVALID_ARGUMENT = 5
};

/* Reference f32 accumulation, output rows [row_begin, row_end) written to
 * out + (row - row_begin) * Wo. nthreads <= 1 runs serially; otherwise rows
 * are split over threads like rayon's into_par_iter over rows. */
int tmo_match_reference(const uint8_t *image, uint32_t W, uint32_t H,
                        const uint8_t *templ, uint32_t w, uint32_t h,
                        const uint8_t *mask, uint32_t mw, uint32_t mh,
                        int method, float *out, uint32_t row_begin,
                        uint32_t row_end, int nthreads);

/* Exact integer sums for every output position. X, Y may be NULL. */
int tmo_sums(const uint8_t *image, uint32_t W, uint32_t H,
             const uint8_t *templ, uint32_t w, uint32_t h,
             const uint8_t *mask, uint64_t *X, uint64_t *Y, uint64_t *tss,
             int nthreads);

/* Exact sums + normalisation in the requested precision. */
int tmo_match_exact(const uint8_t *image, uint32_t W, uint32_t H,
                    const uint8_t *templ, uint32_t w, uint32_t h,
                    const uint8_t *mask, uint32_t mw, uint32_t mh,
                    int method, int precision, float *out, int nthreads);

struct tmo_extremes_s;

/* Fast form of tmo_match_exact for UNMASKED templates of at most 66051
 * pixels (so every X = sum(I*T) fits u32), for the full-size parity checks:
 * X accumulated per output row in u32 with a vectorisable inner loop, Y from
 * the exact u64 integral image of I^2, the same tmo_finish epilogue. The
 * scores equal tmo_match_exact's (tests/test_oracle_fast.py checks this).
 * out (the Wo x Ho map) may be NULL; ext, when not NULL, receives
 * find_extremes of the f32 map (first occurrence in row-major order; the
 * map has no NaN). Returns TMO_ERR_INVALID_ARGUMENT for larger templates. */
int tmo_match_exact_fast(const uint8_t *image, uint32_t W, uint32_t H,
                         const uint8_t *templ, uint32_t w, uint32_t h,
                         int method, int precision, float *out,
                         struct tmo_extremes_s *ext, int nthreads);

/* The same for n unmasked templates of one size (back to back in
 * `templates`) against one image, output rows [row_begin, row_end) only:
 * out (NULL allowed) receives n template-major maps of
 * (row_end - row_begin) x Wo scores, ext (NULL allowed) n records of
 * find_extremes over those rows, locations in full-map coordinates. */
int tmo_many_exact_fast(const uint8_t *image, uint32_t W, uint32_t H,
                        const uint8_t *templates, uint32_t w, uint32_t h,
                        uint32_t n, int method, int precision,
                        uint32_t row_begin, uint32_t row_end, float *out,
                        struct tmo_extremes_s *ext, int nthreads);

/* One output from exact sums (the epilogue the GPU kernels must match). */
float tmo_finish(int method, int precision, uint64_t X, uint64_t Y,
                 uint64_t tss);

typedef struct tmo_extremes_s {
    double max_value, min_value;
    uint32_t max_x, max_y, min_x, min_y;
} tmo_extremes;

/* find_extremes (src/template_matching.rs:479-511) over a row-major image of
 * the given element type code: 0 u8, 1 u16, 2 u32, 3 u64, 4 i8, 5 i16,
 * 6 i32, 7 i64, 8 f32, 9 f64. Values are returned widened to double (exact
 * for every type except 64-bit integers above 2^53; the raw-bits variant
 * below is used for those). */
int tmo_find_extremes(const void *image, uint32_t W, uint32_t H, int type,
                      tmo_extremes *out);

/* Same scan, returning the linear indices of the extremes. */
int tmo_find_extremes_index(const void *image, uint32_t W, uint32_t H,
                            int type, uint64_t *max_index,
                            uint64_t *min_index);

#ifdef __cplusplus
}
#endif
#endif
