// tm_sat.cu -- imageproc's integral_image / integral_squared_image on the
// device (src/integral_image.rs:50-153): a (W+1) x (H+1) table per channel,
// S[y][x][c] = sum of F(x', y')[c] (or its square) over x' < x, y' < y, with a
// zero top row and left column; channels (1 Luma, 3 Rgb, 4 Rgba) interleaved
// like the source pixels.
//
// Element types: u64 (exact for any image that fits in device memory) and
// u32, whose additions wrap modulo 2^32 like the reference's u32 sums in a
// release build; because addition modulo 2^32 is associative, the parallel
// scans below give the reference's sequential result bit for bit.
//
// Two passes over the table: a row scan (one block per row, tiles of 1024
// pixels scanned block-wide and stored through shared memory in contiguous
// runs), then a column scan of the (W+1)*C interleaved columns in place (32
// row segments per block: segment totals, then the rescan with offsets).
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

constexpr int kRowThreads = 256;
constexpr int kPix = 4;                          // pixels per thread per tile
constexpr int kTile = kRowThreads * kPix;        // pixels per tile

// Row pass: each block scans whole rows in tiles of kTile pixels -- a
// per-thread scan of kPix pixels, a block-wide exclusive scan of the thread
// totals per channel, the running carry of the row -- and stages the tile in
// shared memory so that warps store contiguous runs of the table.
template <typename T, bool kSquare, int C>
__global__ void __launch_bounds__(kRowThreads) sat_rows_kernel(const uint8_t* __restrict__ img, uint32_t W,
                                                               uint32_t H, T* __restrict__ sat) {
  __shared__ T s_tile[kTile * C];
  __shared__ T s_warp[C][kRowThreads / 32];
  const uint32_t pitch = (W + 1) * C;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t y = blockIdx.x; y < H; y += gridDim.x) {
    const uint8_t* row = img + (size_t)y * W * C;
    T* out = sat + (size_t)(y + 1) * pitch;
    if (threadIdx.x < C) out[threadIdx.x] = 0;
    T carry[C];
#pragma unroll
    for (int c = 0; c < C; ++c) carry[c] = 0;
    for (uint32_t tile = 0; tile < W; tile += kTile) {
      T pre[kPix][C], acc[C];
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = 0;
#pragma unroll
      for (int j = 0; j < kPix; ++j) {
        const uint32_t x = tile + threadIdx.x * kPix + j;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const T v = x < W ? (T)row[(size_t)x * C + c] : (T)0;
          acc[c] += kSquare ? v * v : v;
          pre[j][c] = acc[c];
        }
      }
      T off[C], tot[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        T incl = acc[c];
        for (int o = 1; o < 32; o <<= 1) {
          const T n = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += n;
        }
        if (lane == 31) s_warp[c][warp] = incl;
        off[c] = incl - acc[c];
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < C; ++c) {
        tot[c] = 0;
        for (int k = 0; k < kRowThreads / 32; ++k) {
          const T wsum = s_warp[c][k];
          if (k < warp) off[c] += wsum;
          tot[c] += wsum;
        }
      }
#pragma unroll
      for (int j = 0; j < kPix; ++j)
#pragma unroll
        for (int c = 0; c < C; ++c) s_tile[(threadIdx.x * kPix + j) * C + c] = carry[c] + off[c] + pre[j][c];
      __syncthreads();
      const uint32_t n = min((uint32_t)kTile, W - tile) * C;
      T* dst = out + (size_t)(tile + 1) * C;
      for (uint32_t e = threadIdx.x; e < n; e += kRowThreads) dst[e] = s_tile[e];
#pragma unroll
      for (int c = 0; c < C; ++c) carry[c] += tot[c];
      __syncthreads();  // s_tile and s_warp are rewritten by the next tile
    }
  }
}

// Column pass: 32 columns x 32 row segments per block; each warp sums its
// segment of 32 columns (coalesced rows), the block turns the segment totals
// into offsets, and each warp rescans its segment adding the offset.
constexpr int kSegs = 32;

template <typename T>
__global__ void __launch_bounds__(32 * kSegs) sat_cols_kernel(uint32_t cols, uint32_t H, T* __restrict__ sat) {
  __shared__ T s_tot[kSegs][33];
  const uint32_t col = blockIdx.x * 32 + (threadIdx.x & 31);
  const int segi = threadIdx.x >> 5;
  const uint32_t seg = (H + kSegs - 1) / kSegs;
  const uint32_t r0 = 1 + segi * seg;
  const uint32_t r1 = min(H + 1, r0 + seg);
  T tot = 0;
  if (col < cols) {
#pragma unroll 8
    for (uint32_t r = r0; r < r1; ++r) tot += sat[(size_t)r * cols + col];
  }
  s_tot[segi][threadIdx.x & 31] = tot;
  __syncthreads();
  T run = 0;
  for (int k = 0; k < segi; ++k) run += s_tot[k][threadIdx.x & 31];
  if (col < cols) {
    // eight rows loaded before any is stored, so the reads overlap instead of
    // waiting on each other through the stores
    uint32_t r = r0;
    for (; r + 8 <= r1; r += 8) {
      T v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = sat[(size_t)(r + k) * cols + col];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        run += v[k];
        sat[(size_t)(r + k) * cols + col] = run;
      }
    }
    for (; r < r1; ++r) {
      T* p = sat + (size_t)r * cols + col;
      run += *p;
      *p = run;
    }
  }
}

template <typename T, bool kSquare, int C>
cudaError_t launch_sat_typed(const uint8_t* img, uint32_t W, uint32_t H, T* sat, cudaStream_t s) {
  const uint32_t cols = (W + 1) * C;
  cudaError_t e = cudaMemsetAsync(sat, 0, sizeof(T) * cols, s);  // top row
  if (e != cudaSuccess || H == 0) return e;
  if (W == 0) return cudaMemsetAsync(sat, 0, sizeof(T) * (size_t)cols * (H + 1), s);
  sat_rows_kernel<T, kSquare, C><<<H < 65535u ? H : 65535u, kRowThreads, 0, s>>>(img, W, H, sat);
  count_launch(kKernelIntegralRows);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  sat_cols_kernel<T><<<(cols + 31) / 32, 32 * kSegs, 0, s>>>(cols, H, sat);
  count_launch(kKernelIntegralCols);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sat_t(const uint8_t* img, uint32_t W, uint32_t H, uint32_t channels, bool squared, T* sat,
                         cudaStream_t s) {
  switch (channels * 2 + (squared ? 1 : 0)) {
    case 2: return launch_sat_typed<T, false, 1>(img, W, H, sat, s);
    case 3: return launch_sat_typed<T, true, 1>(img, W, H, sat, s);
    case 6: return launch_sat_typed<T, false, 3>(img, W, H, sat, s);
    case 7: return launch_sat_typed<T, true, 3>(img, W, H, sat, s);
    case 8: return launch_sat_typed<T, false, 4>(img, W, H, sat, s);
    case 9: return launch_sat_typed<T, true, 4>(img, W, H, sat, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_sat(const uint8_t* img, uint32_t W, uint32_t H, uint32_t channels, bool squared, int bits,
                       void* sat, cudaStream_t s) {
  if (bits == 32) return launch_sat_t<uint32_t>(img, W, H, channels, squared, static_cast<uint32_t*>(sat), s);
  return launch_sat_t<unsigned long long>(img, W, H, channels, squared, static_cast<unsigned long long*>(sat), s);
}

}  // namespace ipb
