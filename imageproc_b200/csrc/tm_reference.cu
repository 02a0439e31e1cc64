// tm_reference.cu -- the reference's f32 arithmetic, replicated on the GPU.
//
// IPB_PRECISION_REFERENCE_F32 reproduces imageproc's scores bit for bit on
// every input, including templates above 258 pixels where the reference's
// sequential f32 sums round. Each output is one dependent chain of f32 adds
// in the reference's order (dy-outer, dx-inner, src/template_matching.rs:
// 410-416 and :447-454) with the reference's per-pixel closure
// (:223, :245-246, :264, :286-287, :305, :328-329, :346, :369-370) and final
// normalisation (:249-250, :290-291, :332-333, :373-374). Every multiply and
// add is an explicitly rounded intrinsic, so nothing is contracted into an
// FMA (the Rust code never fuses). Parallelism comes from independent output
// positions: each thread runs four chains for four adjacent columns.
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

// square_sum / mult_square_sum (:378-386): one sequential f32 sum over the
// template in raw-buffer order, done by a single thread.
__global__ void template_sum_f32_kernel(const uint8_t* __restrict__ tpl,
                                        const uint8_t* __restrict__ mask, size_t n,
                                        float* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float acc = 0.0f;
  for (size_t k = 0; k < n; ++k) {
    const float t = (float)tpl[k];
    if (mask) {
      const float p = __fmul_rn(t, (float)mask[k]);
      acc = __fadd_rn(acc, __fmul_rn(p, p));
    } else {
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
  }
  *out = acc;
}

template <bool kMasked, int kMethod>
__device__ __forceinline__ void step(float& s, float& q, float i, float t, float m) {
  if constexpr (!kMasked) {
    if constexpr (kMethod == kSse || kMethod == kSseNorm) {
      const float d = __fsub_rn(t, i);  // (t - i).powi(2)
      s = __fadd_rn(s, __fmul_rn(d, d));
    } else {
      s = __fadd_rn(s, __fmul_rn(i, t));  // i * t
    }
    if constexpr (kMethod == kSseNorm || kMethod == kCcorrNorm) q = __fadd_rn(q, __fmul_rn(i, i));
  } else {
    if constexpr (kMethod == kSse || kMethod == kSseNorm) {
      const float e = __fmul_rn(__fsub_rn(t, i), m);  // ((t - i) * m).powi(2)
      s = __fadd_rn(s, __fmul_rn(e, e));
    } else {
      s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(t, i), m), m));  // t * i * m * m
    }
    if constexpr (kMethod == kSseNorm || kMethod == kCcorrNorm) {
      const float p = __fmul_rn(i, m);  // (i * m).powi(2)
      q = __fadd_rn(q, __fmul_rn(p, p));
    }
  }
}

template <bool kMasked, int kMethod>
__global__ void __launch_bounds__(128)
reference_kernel(const uint8_t* __restrict__ img, uint32_t W, const uint8_t* __restrict__ tpl,
                 const uint8_t* __restrict__ mask, uint32_t w, uint32_t h, uint32_t Wo,
                 uint32_t Ho, const float* __restrict__ tss_ptr, float* __restrict__ out) {
  const uint32_t x0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (x0 >= Wo) return;
  const uint32_t wlast = W - 1;
  for (uint32_t y = blockIdx.y; y < Ho; y += gridDim.y) {
    float s[4] = {0.f, 0.f, 0.f, 0.f}, q[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t dy = 0; dy < h; ++dy) {
      const uint8_t* ir = img + (size_t)(y + dy) * W;
      const uint8_t* tr = tpl + (size_t)dy * w;
      const uint8_t* mr = kMasked ? mask + (size_t)dy * w : nullptr;
      // columns past the image edge only feed outputs past Wo, which are not
      // stored; clamping keeps their reads in bounds
      float i0 = (float)__ldg(ir + min(x0, wlast));
      float i1 = (float)__ldg(ir + min(x0 + 1, wlast));
      float i2 = (float)__ldg(ir + min(x0 + 2, wlast));
      for (uint32_t dx = 0; dx < w; ++dx) {
        const float i3 = (float)__ldg(ir + min(x0 + 3 + dx, wlast));
        const float t = (float)__ldg(tr + dx);
        const float m = kMasked ? (float)__ldg(mr + dx) : 0.f;
        step<kMasked, kMethod>(s[0], q[0], i0, t, m);
        step<kMasked, kMethod>(s[1], q[1], i1, t, m);
        step<kMasked, kMethod>(s[2], q[2], i2, t, m);
        step<kMasked, kMethod>(s[3], q[3], i3, t, m);
        i0 = i1;
        i1 = i2;
        i2 = i3;
      }
    }
    const float tss = *tss_ptr;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (x0 + k >= Wo) break;
      float r = s[k];
      if constexpr (kMethod == kSseNorm || kMethod == kCcorrNorm) {
        // unmasked: (ii * tss).sqrt(); masked: (tss * im_im).sqrt()
        const float norm = kMasked ? __fsqrt_rn(__fmul_rn(tss, q[k])) : __fsqrt_rn(__fmul_rn(q[k], tss));
        r = norm > 0.0f ? __fdiv_rn(s[k], norm) : s[k];
      }
      out[(size_t)y * Wo + x0 + k] = r;
    }
  }
}

template <bool kMasked>
cudaError_t launch_masked(const MatchArgs& a, const float* tss) {
  const uint32_t Wo = a.W - a.w + 1, Ho = a.H - a.h + 1;
  const int threads = 128;
  const dim3 grid((Wo + 4 * threads - 1) / (4 * threads), Ho < 65535u ? Ho : 65535u);
  timer_begin(a.timer, kKernelReference, a.stream);
  switch (a.method) {
    case kSse:
      reference_kernel<kMasked, kSse><<<grid, threads, 0, a.stream>>>(a.img, a.W, a.tpl, a.mask, a.w, a.h, Wo, Ho, tss, a.out);
      break;
    case kSseNorm:
      reference_kernel<kMasked, kSseNorm><<<grid, threads, 0, a.stream>>>(a.img, a.W, a.tpl, a.mask, a.w, a.h, Wo, Ho, tss, a.out);
      break;
    case kCcorr:
      reference_kernel<kMasked, kCcorr><<<grid, threads, 0, a.stream>>>(a.img, a.W, a.tpl, a.mask, a.w, a.h, Wo, Ho, tss, a.out);
      break;
    default:
      reference_kernel<kMasked, kCcorrNorm><<<grid, threads, 0, a.stream>>>(a.img, a.W, a.tpl, a.mask, a.w, a.h, Wo, Ho, tss, a.out);
      break;
  }
  count_launch(kKernelReference);
  timer_end(a.timer, a.stream);
  return cudaGetLastError();
}

}  // namespace

size_t reference_scratch_bytes(const MatchArgs&) { return 256; }

cudaError_t launch_reference(const MatchArgs& a, void* scratch) {
  float* tss = static_cast<float*>(scratch);
  template_sum_f32_kernel<<<1, 32, 0, a.stream>>>(a.tpl, a.mask, (size_t)a.w * a.h, tss);
  count_launch(kKernelTemplateSumF32);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return a.mask ? launch_masked<true>(a, tss) : launch_masked<false>(a, tss);
}

}  // namespace ipb
