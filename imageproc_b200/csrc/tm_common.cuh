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

__host__ __device__ constexpr bool method_is_sse(int m) { return m == kSse || m == kSseNorm; }
__host__ __device__ constexpr bool method_is_norm(int m) { return m == kSseNorm || m == kCcorrNorm; }

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

// Exact u32 -> double without a conversion instruction: the bits
// 0x43300000:u are the double 2^52 + u.
__device__ __forceinline__ double u32_to_double(uint32_t u) {
  return __dsub_rn(__hiloint2double(0x43300000, (int)u), 4503599627370496.0);
}

// RN_f32(RN_d(s / RN_d(sqrt(P)))) for an integer s < 2^32 and a double P in
// [1, 2^64], the EXACT_FP64 normalisation, computed through a filter:
//  * r0 = rsqrtf(P rounded down to f32): relative error d below 2^-21.6
//    (rsqrtf is accurate to 2 ulp, 2^-22; the truncation adds 2^-24);
//  * one Newton-Raphson step for the reciprocal square root in double,
//    r1 = r0 + r0 (1 - P r0^2) / 2, leaves a relative error of about
//    1.5 d^2 (2^-42.6) plus a few double roundings, below 2^-40.5;
//  * a = s r1 then differs from the correctly rounded quotient q by less
//    than 2^-40.4 |a|, i.e. fewer than 2^13 units in the last place of a.
// Rounding to f32 is monotone, so when the 29 mantissa bits of a that f32
// drops are more than 2^16 units away from the rounding midpoint 2^28, q
// rounds to the same f32 as a, which is then formed from a's bits (truncate,
// plus one when above the midpoint; a lies in f32's normal range). Otherwise
// (about one value in 4096) the quotient is formed by the IEEE-rounded
// sqrt and divide themselves, out of line to keep unrolled callers small.
static __device__ __noinline__ float norm_quotient_fp64_ieee(uint32_t s, double P) {
  return __double2float_rn(__ddiv_rn(u32_to_double(s), __dsqrt_rn(P)));
}

__device__ __forceinline__ float norm_quotient_fp64(uint32_t s, double P) {
  if (s == 0u) return 0.0f;
  const uint32_t phi = (uint32_t)__double2hiint(P), plo = (uint32_t)__double2loint(P);
  const float pf = __uint_as_float(((phi - (896u << 20)) << 3) | (plo >> 29));
  const uint32_t ru = __float_as_uint(rsqrtf(pf));
  const double r0 = __hiloint2double((int)((ru >> 3) + (896u << 20)), (int)(ru << 29));
  const double e = __fma_rn(-__dmul_rn(P, r0), r0, 1.0);
  const double r1 = __fma_rn(r0, __dmul_rn(e, 0.5), r0);
  const double a = __dmul_rn(u32_to_double(s), r1);
  const uint32_t ahi = (uint32_t)__double2hiint(a), alo = (uint32_t)__double2loint(a);
  const uint32_t dropped = alo & 0x1FFFFFFFu;
  if (dropped - (0x10000000u - 0x10000u) < 0x20000u) return norm_quotient_fp64_ieee(s, P);
  return __uint_as_float((((ahi - (896u << 20)) << 3) | (alo >> 29)) + (dropped >> 28));
}

// 1/sqrt(v) for an integer 1 <= v < 2^32 in double, to within about 2^-51
// relative: rsqrtf of v rounded to f32 (relative error below 2^-21.6), then
// two Newton-Raphson steps for the reciprocal square root (each squares the
// error, down to the double roundings).
__device__ __forceinline__ double rsqrt_u32(uint32_t v) {
  const double vd = u32_to_double(v);
  double r = (double)rsqrtf(__uint2float_rn(v));
  r = __fma_rn(r, __dmul_rn(__fma_rn(-__dmul_rn(vd, r), r, 1.0), 0.5), r);
  return __fma_rn(r, __dmul_rn(__fma_rn(-__dmul_rn(vd, r), r, 1.0), 0.5), r);
}

// EXACT_FP64 normalisation through precomputed reciprocal roots:
// w = rsqrt_u32(Y) * rsqrt_u32(T) (0 when Y or T is 0). a = s * w is within
// 2^-49 relative of s / sqrt(Y T), and the quotient q = RN_d(s / RN_d(sqrt(
// RN_d(Y T)))) within 2^-51, so a is fewer than 2^5 units in its last place
// from q and the midpoint test of norm_quotient_fp64 (2^16 units) decides
// RN_f32(q); undecided values take the IEEE-rounded sqrt and divide.
__device__ __forceinline__ float norm_quotient_fp64_w(uint32_t s, double w, uint32_t Y, uint32_t T) {
  if (w == 0.0) return __uint2float_rn(s);  // zero norm
  if (s == 0u) return 0.0f;
  const double a = __dmul_rn(u32_to_double(s), w);
  const uint32_t ahi = (uint32_t)__double2hiint(a), alo = (uint32_t)__double2loint(a);
  const uint32_t dropped = alo & 0x1FFFFFFFu;
  if (dropped - (0x10000000u - 0x10000u) < 0x20000u)
    return norm_quotient_fp64_ieee(s, __dmul_rn(u32_to_double(Y), u32_to_double(T)));
  return __uint_as_float((((ahi - (896u << 20)) << 3) | (alo >> 29)) + (dropped >> 28));
}

// The common case of norm_quotient_fp64_w without branches, for epilogues
// that score many values independently: w > 0 is a normal double.
// a = RN(s w) comes from one fused multiply-add, fma(2^52 + s, w, -2^52 w):
// 2^52 + s is s's bits under the exponent of 2^52 (exact for s < 2^32),
// -2^52 w is w with 52 added to its exponent and the sign set (one integer
// add on the high word), and the fma rounds the exact s w once -- the same
// double as RN(RN_d(s) * w). The midpoint window is 2^8 units of a's last
// place on either side: a is fewer than 2^5 units from q (the bound of
// norm_quotient_fp64_w), so a value outside the window rounds to the same
// f32 as q. `undecided` is set when the result must come from
// norm_quotient_fp64_w instead (a inside the window). s == 0 gives a == 0, whose high word is clamped up to the bias
// difference so that the formed bits are those of +0.0f, the zero-score rule.
__device__ __forceinline__ uint32_t norm_bits_fp64_fast(uint32_t s, double w, bool& undecided) {
  const double d = __hiloint2double(0x43300000, (int)s);
  const double nc = __hiloint2double((int)((uint32_t)__double2hiint(w) + 0x83400000u), __double2loint(w));
  const double a = __fma_rn(d, w, nc);
  const uint32_t ahi = (uint32_t)__double2hiint(a), alo = (uint32_t)__double2loint(a);
  const uint32_t dropped = alo & 0x1FFFFFFFu;
  undecided |= dropped - (0x10000000u - 0x100u) < 0x200u;
  const uint32_t hi = max(ahi, 896u << 20);  // a == 0: every formed bit is zero
  return (((hi - (896u << 20)) << 3) | (alo >> 29)) + (dropped >> 28);
}

// finish_score for callers whose X, Y and TSS are all below 2^31 (templates
// of at most 33025 pixels): the integer score fits in 32 bits, and SSE's
// Y + TSS - 2X is exact in wrapping u32 arithmetic because the true result
// is below 2^32. Same results as finish_score (the FP64 quotient through
// norm_quotient_fp64).
__device__ __forceinline__ float finish_score32(int method, int precision, uint32_t X, uint32_t Y,
                                                uint32_t tss) {
  const uint32_t score = method_is_sse(method) ? (Y + tss - 2u * X) : X;
  if (!method_is_norm(method)) return __uint2float_rn(score);
  if (precision == IPB_PRECISION_EXACT_FP64) {
    if (Y == 0u || tss == 0u) return __uint2float_rn(score);  // zero norm
    return norm_quotient_fp64(score, __dmul_rn(u32_to_double(Y), u32_to_double(tss)));
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
