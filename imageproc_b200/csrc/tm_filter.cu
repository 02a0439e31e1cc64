// tm_filter.cu -- imageproc's filter_clamped on the device (src/filter/mod.rs:
// 29-70, :202-212): the 2-D correlation of a u8 image (1, 3 or 4 interleaved
// channels) with a row-major kernel, padded by continuity (coordinates clamped
// to the image), accumulated per channel in the kernel's type and clamped to
// the output type by the reference's Clamp (src/definitions.rs:114-190).
//
// The reference's arithmetic is kept exactly: for each output pixel the sum
// runs k_y outer, k_x inner, acc = acc + (K)pixel * weight with one rounding
// per multiply and per add for f32 kernels (explicitly rounded intrinsics, no
// contraction) and wrapping two's-complement arithmetic for i32 kernels (a
// release build). Each thread computes one output pixel in that order; a
// block stages its 32 x 8 output tile's input window (clamped) and the kernel
// in shared memory.
#include <type_traits>

#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

__device__ __forceinline__ uint32_t align_up_dev(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

constexpr int kTX = 32, kTY = 8;
constexpr uint32_t kMaxTileKernel = 64;  // kernels up to 64 x 64 use the shared-memory tile

// Clamp<K> for S (src/definitions.rs:119-190): values at or above the maximum
// (and NaN) give the maximum, values at or below the minimum the minimum,
// the rest convert (f32 -> integer truncates toward zero).
template <typename S, typename K>
__device__ __forceinline__ S clamp_to(K x) {
  if constexpr (std::is_same<S, K>::value) {
    return x;
  } else {
    constexpr K hi = std::is_same<S, uint8_t>::value ? (K)255 : std::is_same<S, uint16_t>::value ? (K)65535 : (K)32767;
    constexpr K lo = std::is_same<S, int16_t>::value ? (K)-32768 : (K)0;
    if (x < hi) return x > lo ? (S)x : (S)lo;
    return (S)hi;
  }
}

template <typename K>
__device__ __forceinline__ K mac(K acc, uint8_t pix, K w) {
  if constexpr (std::is_same<K, float>::value) {
    return __fadd_rn(acc, __fmul_rn((float)pix, w));
  } else {  // i32, wrapping
    return (int32_t)((uint32_t)acc + (uint32_t)pix * (uint32_t)w);
  }
}

template <int C, typename K, typename S>
__global__ void __launch_bounds__(kTX* kTY) filter_tile_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t H,
                                                              const K* __restrict__ kern, uint32_t kw, uint32_t kh,
                                                              S* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t smem[];
  K* s_k = reinterpret_cast<K*>(smem);
  uint8_t* s_img = smem + align_up_dev(kw * kh * sizeof(K), 16);
  const uint32_t tw = kTX + kw - 1, th = kTY + kh - 1;
  const int x0 = (int)(blockIdx.x * kTX) - (int)(kw / 2), y0 = (int)(blockIdx.y * kTY) - (int)(kh / 2);
  const uint32_t tid = threadIdx.y * kTX + threadIdx.x;
  for (uint32_t i = tid; i < kw * kh; i += kTX * kTY) s_k[i] = kern[i];
  for (uint32_t i = tid; i < tw * th; i += kTX * kTY) {
    const int ty = (int)(i / tw), tx = (int)(i % tw);
    const int yy = min((int)H - 1, max(0, y0 + ty)), xx = min((int)W - 1, max(0, x0 + tx));
#pragma unroll
    for (int c = 0; c < C; ++c) s_img[i * C + c] = img[((size_t)yy * W + xx) * C + c];
  }
  __syncthreads();
  const uint32_t x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
  if (x >= W || y >= H) return;
  K acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0;
  for (uint32_t ky = 0; ky < kh; ++ky) {
    const uint8_t* row = s_img + ((threadIdx.y + ky) * tw + threadIdx.x) * C;
    const K* krow = s_k + ky * kw;
    for (uint32_t kx = 0; kx < kw; ++kx) {
      const K w = krow[kx];
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = mac(acc[c], row[kx * C + c], w);
    }
  }
#pragma unroll
  for (int c = 0; c < C; ++c) out[((size_t)y * W + x) * C + c] = clamp_to<S>(acc[c]);
}

// Kernels wider or taller than the tile path takes: the same loop with
// clamped coordinates read through the cache.
template <int C, typename K, typename S>
__global__ void __launch_bounds__(kTX* kTY) filter_global_kernel(const uint8_t* __restrict__ img, uint32_t W,
                                                                uint32_t H, const K* __restrict__ kern, uint32_t kw,
                                                                uint32_t kh, S* __restrict__ out) {
  const uint32_t x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
  if (x >= W || y >= H) return;
  K acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0;
  for (uint32_t ky = 0; ky < kh; ++ky) {
    const long long yy = min((long long)H - 1, max(0ll, (long long)y + ky - kh / 2));
    for (uint32_t kx = 0; kx < kw; ++kx) {
      const long long xx = min((long long)W - 1, max(0ll, (long long)x + kx - kw / 2));
      const K w = __ldg(kern + (size_t)ky * kw + kx);
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = mac(acc[c], __ldg(img + ((size_t)yy * W + xx) * C + c), w);
    }
  }
#pragma unroll
  for (int c = 0; c < C; ++c) out[((size_t)y * W + x) * C + c] = clamp_to<S>(acc[c]);
}

template <int C, typename K, typename S>
cudaError_t launch_filter_t(const uint8_t* img, uint32_t W, uint32_t H, const void* kern, uint32_t kw, uint32_t kh,
                            void* out, cudaStream_t s) {
  const dim3 grid((W + kTX - 1) / kTX, (H + kTY - 1) / kTY), block(kTX, kTY);
  if (grid.y > 65535u) return cudaErrorInvalidValue;
  const K* k = static_cast<const K*>(kern);
  S* o = static_cast<S*>(out);
  if (kw <= kMaxTileKernel && kh <= kMaxTileKernel) {
    const size_t smem = align_up((size_t)kw * kh * sizeof(K), 16) + (size_t)(kTX + kw - 1) * (kTY + kh - 1) * C;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(filter_tile_kernel<C, K, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
    }
    filter_tile_kernel<C, K, S><<<grid, block, smem, s>>>(img, W, H, k, kw, kh, o);
  } else {
    filter_global_kernel<C, K, S><<<grid, block, 0, s>>>(img, W, H, k, kw, kh, o);
  }
  count_launch(kKernelFilter);
  return cudaGetLastError();
}

template <int C>
cudaError_t launch_filter_c(const uint8_t* img, uint32_t W, uint32_t H, const void* kern, int ktype, uint32_t kw,
                            uint32_t kh, int otype, void* out, cudaStream_t s) {
  if (ktype == IPB_KERNEL_TYPE_F32) {
    switch (otype) {
      case IPB_ELEM_U8: return launch_filter_t<C, float, uint8_t>(img, W, H, kern, kw, kh, out, s);
      case IPB_ELEM_U16: return launch_filter_t<C, float, uint16_t>(img, W, H, kern, kw, kh, out, s);
      case IPB_ELEM_F32: return launch_filter_t<C, float, float>(img, W, H, kern, kw, kh, out, s);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (otype) {
    case IPB_ELEM_U8: return launch_filter_t<C, int32_t, uint8_t>(img, W, H, kern, kw, kh, out, s);
    case IPB_ELEM_U16: return launch_filter_t<C, int32_t, uint16_t>(img, W, H, kern, kw, kh, out, s);
    case IPB_ELEM_I16: return launch_filter_t<C, int32_t, int16_t>(img, W, H, kern, kw, kh, out, s);
    case IPB_ELEM_I32: return launch_filter_t<C, int32_t, int32_t>(img, W, H, kern, kw, kh, out, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

bool filter_types_supported(int ktype, int otype) {
  if (ktype == IPB_KERNEL_TYPE_F32) return otype == IPB_ELEM_U8 || otype == IPB_ELEM_U16 || otype == IPB_ELEM_F32;
  if (ktype == IPB_KERNEL_TYPE_I32)
    return otype == IPB_ELEM_U8 || otype == IPB_ELEM_U16 || otype == IPB_ELEM_I16 || otype == IPB_ELEM_I32;
  return false;
}

cudaError_t launch_filter(const uint8_t* img, uint32_t W, uint32_t H, uint32_t channels, const void* kern, int ktype,
                          uint32_t kw, uint32_t kh, int otype, void* out, cudaStream_t s) {
  if (W == 0 || H == 0) return cudaSuccess;
  switch (channels) {
    case 1: return launch_filter_c<1>(img, W, H, kern, ktype, kw, kh, otype, out, s);
    case 3: return launch_filter_c<3>(img, W, H, kern, ktype, kw, kh, otype, out, s);
    case 4: return launch_filter_c<4>(img, W, H, kern, ktype, kw, kh, otype, out, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ipb
