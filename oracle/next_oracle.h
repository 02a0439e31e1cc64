/*
 * next_oracle.h -- CPU oracle for the rows next to the template-matching path:
 * imageproc's integral images and non-maximum suppression.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels, called by the
 * test-suite and nothing else.
 *
 * Parity status: pinned against the reference's known-answer tests
 * (src/integral_image.rs:471-567, src/suppress.rs:209-258), extracted as text
 * into tests/golden/reference_next_tests.json, and against the naive
 * definition of suppress_non_maximum the reference's own tests hold
 * (src/suppress.rs:274-318).
 */
#ifndef NEXT_ORACLE_H
#define NEXT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* integral_image / integral_squared_image (src/integral_image.rs:98-153): for
 * each row a running sum of F (or F^2) in T arithmetic, added to the entry
 * above; (W+1) x (H+1) x C table, zero top row and left column. The u32 form
 * wraps modulo 2^32 like the reference's u32 arithmetic in a release build. */
void nxo_integral_u32(const uint8_t *img, uint32_t W, uint32_t H, uint32_t C, int square, uint32_t *out);
void nxo_integral_u64(const uint8_t *img, uint32_t W, uint32_t H, uint32_t C, int square, uint64_t *out);

/* suppress_non_maximum (src/suppress.rs:10-77, contains_greater_value
 * :82-107) on order-preserving u64 keys of the pixel values: keep[y*W + x] = 1
 * where the reference writes the pixel's value, 0 where it leaves zero. */
void nxo_suppress_non_maximum(const uint64_t *keys, uint32_t W, uint32_t H, uint32_t radius, uint8_t *keep);

/* The naive definition the reference's tests compare against
 * (suppress_non_maximum_reference, src/suppress.rs:274-318). */
void nxo_suppress_non_maximum_naive(const uint64_t *keys, uint32_t W, uint32_t H, uint32_t radius,
                                    uint8_t *keep);

/* local_maxima (src/suppress.rs:111-173) of n scored points: writes the
 * input indices of the points the reference returns, in its order (sorted by
 * (y, x), stable), and returns their count. */
uint32_t nxo_local_maxima(const uint32_t *xs, const uint32_t *ys, const float *scores, uint32_t n,
                          uint32_t radius, uint32_t *out_idx);

/* filter_clamped (src/filter/mod.rs:202-212 through filter :29-70,
 * accumulate :407-416, Clamp src/definitions.rs:119-190): kernel_type 0 = f32,
 * 1 = i32; out_type uses the library's element codes (0 u8, 1 u16, 5 i16,
 * 6 i32, 8 f32). */
void nxo_filter_clamped(const uint8_t *img, uint32_t W, uint32_t H, uint32_t C, const void *kernel,
                        int kernel_type, uint32_t kw, uint32_t kh, int out_type, void *out);

#ifdef __cplusplus
}
#endif
#endif
