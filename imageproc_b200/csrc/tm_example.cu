// tm_example.cu -- the workflow of imageproc's examples/template_matching.rs
// (:122-190) as a device pipeline: crop the template (copy_sub_image :78-92),
// match it (run_match_template :100-134), rescale the score map to u8 over its
// own range (convert_to_gray_image :63-76), pad it to the image size and draw
// the crop's outline in green (draw_green_rect :94-98). Decoding and encoding
// the PNG files stays on the host.
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

constexpr int kThreads = 256;

__global__ void crop_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t x, uint32_t y, uint32_t w,
                            uint32_t h, uint8_t* __restrict__ out) {
  const size_t n = (size_t)w * h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t sy = (uint32_t)(i / w), sx = (uint32_t)(i % w);
    out[i] = img[(size_t)(y + sy) * W + x + sx];
  }
}

// Order key of an f32 (total order on the bit patterns).
__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fkey_value(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// keys[0] = key(lo), keys[1] = key(hi), seeded with +inf and -inf. The
// reference scans with `*p < lo` and `*p > hi`, so a NaN never becomes an
// extreme; fminf / fmaxf skip NaN the same way. Which of two equal zeros wins
// may differ from the scan, and no pixel depends on it: x - lo and hi - lo
// are the same up to the sign of a zero, which the u8 conversion erases.
__global__ void range_init_kernel(uint32_t* keys) {
  keys[0] = 0xFF800000u;  // key(+inf)
  keys[1] = 0x007FFFFFu;  // key(-inf)
}

__global__ void __launch_bounds__(kThreads) range_kernel(const float* __restrict__ v, size_t n,
                                                         uint32_t* __restrict__ keys) {
  float lo = __int_as_float(0x7F800000), hi = __int_as_float(0xFF800000);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float p = v[i];
    lo = fminf(lo, p);
    hi = fmaxf(hi, p);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ float s_lo[kThreads / 32], s_hi[kThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kThreads / 32; ++k) {
      lo = fminf(lo, s_lo[k]);
      hi = fmaxf(hi, s_hi[k]);
    }
    atomicMin(&keys[0], fkey(lo));
    atomicMax(&keys[1], fkey(hi));
  }
}

// `(255.0 * (x - lo) / range) as u8`: f32 operations in the reference's order,
// then Rust's saturating cast (NaN -> 0, truncation toward zero, clamp).
__device__ __forceinline__ uint32_t scale_u8(float x, float lo, float range) {
  const float s = __fdiv_rn(__fmul_rn(255.0f, __fsub_rn(x, lo)), range);
  if (!(s > 0.0f)) return 0u;  // NaN, zero and negatives
  if (s >= 255.0f) return 255u;
  return (uint32_t)s;
}

struct Render {
  const uint8_t* gray;  // source pixels, or null: the padded, rescaled score map
  const float* map;
  uint32_t Wo, Ho, px, py;  // map size and its offset in the W x H canvas
  const uint32_t* keys;     // the map's range
  uint32_t W, H;
  int32_t left, top, right, bottom;  // outline drawn in green
  uint8_t* rgb;                      // W x H x 3
};

// Four pixels per thread: 12 bytes, three aligned 32-bit stores.
__global__ void __launch_bounds__(kThreads) render_kernel(const Render r) {
  const size_t n = (size_t)r.W * r.H;
  float lo = 0.f, range = 0.f;
  if (!r.gray) {
    lo = fkey_value(r.keys[0]);
    range = __fsub_rn(fkey_value(r.keys[1]), lo);
  }
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; 4 * q < n; q += (size_t)gridDim.x * blockDim.x) {
    uint8_t px[12];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t i = 4 * q + k;
      uint32_t v = 0;
      int32_t x = 0, y = 0;
      if (i < n) {
        y = (int32_t)(i / r.W);
        x = (int32_t)(i % r.W);
        if (r.gray) {
          v = r.gray[i];
        } else {
          const uint32_t mx = (uint32_t)x - r.px, my = (uint32_t)y - r.py;  // wraps below the offset
          if (mx < r.Wo && my < r.Ho) v = scale_u8(r.map[(size_t)my * r.Wo + mx], lo, range);
        }
      }
      const bool edge = ((y == r.top || y == r.bottom) && x >= r.left && x <= r.right) ||
                        ((x == r.left || x == r.right) && y >= r.top && y <= r.bottom);
      px[3 * k] = edge ? 0 : (uint8_t)v;
      px[3 * k + 1] = edge ? 255 : (uint8_t)v;
      px[3 * k + 2] = edge ? 0 : (uint8_t)v;
    }
    uint8_t* dst = r.rgb + 12 * q;
    if (4 * q + 4 <= n) {
      uint32_t* d4 = reinterpret_cast<uint32_t*>(dst);
#pragma unroll
      for (int k = 0; k < 3; ++k)
        d4[k] = px[4 * k] | (px[4 * k + 1] << 8) | (px[4 * k + 2] << 16) | ((uint32_t)px[4 * k + 3] << 24);
    } else {
      for (size_t k = 0; k < 3 * (n - 4 * q); ++k) dst[k] = px[k];
    }
  }
}

uint32_t grid_for(size_t n) {
  const size_t g = (n + kThreads - 1) / kThreads;
  return (uint32_t)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

cudaError_t launch_crop(const uint8_t* img, uint32_t W, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                        uint8_t* out, cudaStream_t s) {
  if (!w || !h) return cudaSuccess;
  crop_kernel<<<grid_for((size_t)w * h), kThreads, 0, s>>>(img, W, x, y, w, h, out);
  count_launch(kKernelExample);
  return cudaGetLastError();
}

cudaError_t launch_map_range(const float* map, size_t n, uint32_t* keys, cudaStream_t s) {
  range_init_kernel<<<1, 1, 0, s>>>(keys);
  count_launch(kKernelExample);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !n) return e;
  range_kernel<<<grid_for(n), kThreads, 0, s>>>(map, n, keys);
  count_launch(kKernelExample);
  return cudaGetLastError();
}

cudaError_t launch_render(const uint8_t* gray, const float* map, uint32_t Wo, uint32_t Ho, uint32_t px,
                          uint32_t py, const uint32_t* keys, uint32_t W, uint32_t H, int32_t left, int32_t top,
                          int32_t right, int32_t bottom, uint8_t* rgb, cudaStream_t s) {
  const size_t n = (size_t)W * H;
  if (!n) return cudaSuccess;
  const Render r{gray, map, Wo, Ho, px, py, keys, W, H, left, top, right, bottom, rgb};
  render_kernel<<<grid_for((n + 3) / 4), kThreads, 0, s>>>(r);
  count_launch(kKernelExample);
  return cudaGetLastError();
}

}  // namespace ipb
