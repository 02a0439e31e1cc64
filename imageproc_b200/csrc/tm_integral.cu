// tm_integral.cu -- u64 integral images (summed-area tables) on the device.
//
// Layout of imageproc's integral_image / integral_squared_image
// (src/integral_image.rs:11-22, :50, :89): one row and one column larger than
// the source, S[y][x] = sum of F(x', y') for x' < x, y' < y, so the top row and
// left column are zero. The window sum over [x, x+w) x [y, y+h) is
// S[y+h][x+w] - S[y][x+w] - S[y+h][x] + S[y][x], exact in u64 for any image
// that fits in device memory (255^2 * 2^32 < 2^64).
//
// Two passes: a row scan (one block per row) writes the row prefix sums, then
// a column scan adds the column prefixes in place. Both passes are HBM-bound
// streams over the (H+1) x (W+1) x 8 byte table.
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {

size_t integral_bytes(uint32_t W, uint32_t H) {
  return align_up((size_t)(W + 1) * (H + 1) * sizeof(unsigned long long), 256);
}

template <bool kSquare>
__global__ void __launch_bounds__(256) integral_rows_kernel(const uint8_t* __restrict__ img,
                                                            uint32_t W, uint32_t H,
                                                            unsigned long long* __restrict__ sat) {
  __shared__ unsigned long long s_warp[8];
  const uint32_t pitch = W + 1;
  const uint32_t seg = (W + blockDim.x - 1) / blockDim.x;
  for (uint32_t y = blockIdx.x; y < H; y += gridDim.x) {
    const uint8_t* row = img + (size_t)y * W;
    unsigned long long* out = sat + (size_t)(y + 1) * pitch;
    const uint32_t x0 = threadIdx.x * seg;
    const uint32_t x1 = min(W, x0 + seg);
    unsigned long long local = 0;
    for (uint32_t x = x0; x < x1; ++x) {
      const uint32_t v = row[x];
      local += kSquare ? v * v : v;
    }
    // block-wide exclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = local;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long n = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += n;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    unsigned long long base = 0;
    for (int k = 0; k < warp; ++k) base += s_warp[k];
    unsigned long long run = base + incl - local;
    for (uint32_t x = x0; x < x1; ++x) {
      const uint32_t v = row[x];
      run += kSquare ? v * v : v;
      out[x + 1] = run;
    }
    if (threadIdx.x == 0) out[0] = 0;
    __syncthreads();
  }
}

// 32 columns x 8 row segments per block; each thread scans its segment of one
// column twice (segment total, then the prefix with the segment's offset).
__global__ void __launch_bounds__(256) integral_cols_kernel(uint32_t W, uint32_t H,
                                                            unsigned long long* __restrict__ sat) {
  __shared__ unsigned long long s_tot[8][32];
  const uint32_t pitch = W + 1;
  const uint32_t col = blockIdx.x * 32 + (threadIdx.x & 31);
  const int segi = threadIdx.x >> 5;
  const uint32_t seg = (H + 7) / 8;
  const uint32_t r0 = 1 + segi * seg;
  const uint32_t r1 = min(H + 1, r0 + seg);
  unsigned long long tot = 0;
  if (col < pitch)
    for (uint32_t r = r0; r < r1; ++r) tot += sat[(size_t)r * pitch + col];
  s_tot[segi][threadIdx.x & 31] = tot;
  __syncthreads();
  unsigned long long run = 0;
  for (int k = 0; k < segi; ++k) run += s_tot[k][threadIdx.x & 31];
  if (col < pitch)
    for (uint32_t r = r0; r < r1; ++r) {
      unsigned long long* p = sat + (size_t)r * pitch + col;
      run += *p;
      *p = run;
    }
}

template <bool kSquare>
static cudaError_t launch_integral_impl(const uint8_t* img, uint32_t W, uint32_t H,
                                        unsigned long long* sat, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(sat, 0, sizeof(unsigned long long) * (W + 1), s);
  if (e != cudaSuccess || H == 0) return e;
  if (W == 0) {
    // one zero column
    return cudaMemsetAsync(sat, 0, sizeof(unsigned long long) * (size_t)(H + 1), s);
  }
  const unsigned rows_grid = H < 65535u ? H : 65535u;
  integral_rows_kernel<kSquare><<<rows_grid, 256, 0, s>>>(img, W, H, sat);
  count_launch(kKernelIntegralRows);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  integral_cols_kernel<<<(W + 1 + 31) / 32, 256, 0, s>>>(W, H, sat);
  count_launch(kKernelIntegralCols);
  return cudaGetLastError();
}

cudaError_t launch_integral_squared(const uint8_t* img, uint32_t W, uint32_t H,
                                    unsigned long long* sat, cudaStream_t s) {
  return launch_integral_impl<true>(img, W, H, sat, s);
}

cudaError_t launch_integral(const uint8_t* img, uint32_t W, uint32_t H,
                            unsigned long long* sat, cudaStream_t s) {
  return launch_integral_impl<false>(img, W, H, sat, s);
}

}  // namespace ipb
