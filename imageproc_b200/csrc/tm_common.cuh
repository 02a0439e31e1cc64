// tm_common.cuh -- shared device helpers for the template-matching kernels.
//
// Score arithmetic follows imageproc 0.27.0 src/template_matching.rs: every
// method is expressed through three exact integer sums per output position
//   X   = sum I*U   (U = T unmasked, T*m^2 masked)
//   Y   = sum I^2*V (V = 1 unmasked, m^2 masked)
//   TSS = sum (T*m)^2 (per template)
// so that CrossCorrelation = X, SumOfSquaredErrors = Y - 2X + TSS and the
// normalised methods divide by sqrt(Y * TSS) (doc math :12-62, closures
// :219-375).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "imageproc_b200.h"

namespace ipb {

enum Method : int {
  kSse = IPB_SUM_OF_SQUARED_ERRORS,
  kSseNorm = IPB_SUM_OF_SQUARED_ERRORS_NORMALIZED,
  kCcorr = IPB_CROSS_CORRELATION,
  kCcorrNorm = IPB_CROSS_CORRELATION_NORMALIZED,
};

__host__ __device__ inline bool method_is_sse(int m) { return m == kSse || m == kSseNorm; }
__host__ __device__ inline bool method_is_norm(int m) { return m == kSseNorm || m == kCcorrNorm; }

// One output value from the exact sums. EXACT_FP64: sqrt and divide in
// double, one rounding to f32. EXACT_F32: the reference's f32 normalisation
// `(ii * tss).sqrt()`, `score / norm` (:249-250) on the exact sums. The zero
// norm rule `if norm > 0.0 { score / norm } else { score }` is kept in both.
// Every operation is an explicitly rounded intrinsic so the compiler cannot
// contract or reorder it; the CPU oracle performs the same IEEE operations.
__device__ __forceinline__ float finish_score(int method, int precision, unsigned long long X,
                                              unsigned long long Y, unsigned long long tss) {
  const unsigned long long score = method_is_sse(method) ? (Y + tss - 2ull * X) : X;
  if (!method_is_norm(method)) return __ull2float_rn(score);
  if (precision == IPB_PRECISION_EXACT_FP64) {
    const double n = __dsqrt_rn(__dmul_rn(__ull2double_rn(Y), __ull2double_rn(tss)));
    return n > 0.0 ? __double2float_rn(__ddiv_rn(__ull2double_rn(score), n))
                   : __ull2float_rn(score);
  }
  const float s = __ull2float_rn(score);
  const float n = __fsqrt_rn(__fmul_rn(__ull2float_rn(Y), __ull2float_rn(tss)));
  return n > 0.0f ? __fdiv_rn(s, n) : s;
}

// finish_score for callers whose X, Y and TSS are all below 2^31 (templates
// of at most 33025 pixels): the integer score fits in 32 bits, and SSE's
// Y + TSS - 2X is exact in wrapping u32 arithmetic because the true result
// is below 2^32. Same roundings as finish_score.
__device__ __forceinline__ float finish_score32(int method, int precision, uint32_t X, uint32_t Y,
                                                uint32_t tss) {
  const uint32_t score = method_is_sse(method) ? (Y + tss - 2u * X) : X;
  if (!method_is_norm(method)) return __uint2float_rn(score);
  if (precision == IPB_PRECISION_EXACT_FP64) {
    const double n = __dsqrt_rn(__dmul_rn(__uint2double_rn(Y), __uint2double_rn(tss)));
    return n > 0.0 ? __double2float_rn(__ddiv_rn(__uint2double_rn(score), n)) : __uint2float_rn(score);
  }
  const float s = __uint2float_rn(score);
  const float n = __fsqrt_rn(__fmul_rn(__uint2float_rn(Y), __uint2float_rn(tss)));
  return n > 0.0f ? __fdiv_rn(s, n) : s;
}

__device__ __forceinline__ uint32_t dp4a_u8(uint32_t a, uint32_t b, uint32_t c) {
  return __dp4a(a, b, c);
}

// Bytes s..s+3 of the 8-byte little-endian value (hi:lo).
template <int S>
__device__ __forceinline__ uint32_t funnel_bytes(uint32_t lo, uint32_t hi) {
  if constexpr (S == 0) return lo;
  else return __byte_perm(lo, hi, (S) | ((S + 1) << 4) | ((S + 2) << 8) | ((S + 3) << 12));
}

}  // namespace ipb
