// tm_suppress.cu -- imageproc's non-maximum suppression on the device
// (src/suppress.rs).
//
// suppress_non_maximum (:10-107) keeps a pixel's value when it is the
// greatest in the (2r+1) x (2r+1) window centred on it (clipped to the image)
// and writes zero elsewhere; among equal values the pixel with the
// lexicographically smaller (x, y) wins. The reference finds this with a grid
// of (r+1)-cells; the kept set is exactly the per-pixel rule (its own tests
// check that against a naive implementation, :274-318), which is separable:
// "greatest" is the maximum under the total order (value, then (x, y)
// reversed), and the window maximum of a rectangle is the column maximum of
// row maxima. So:
//   row pass:    for every pixel, the column x' in [x-r, x+r] holding the row
//                window's winner (largest value, smallest x' among equals);
//   column pass: for every pixel, the winner of the column window over
//                those row winners (largest value, then smallest (x', y'));
//                the pixel keeps its value iff it is that winner.
// Values compare through order-preserving u64 keys, so one kernel serves
// every integer type (and f32 score maps, where NaN compares above numbers).
//
// local_maxima (:111-173) works on a list of scored points: stable sort by
// (y, x) (CUB radix sort), per-row start offsets, then one thread per point
// runs the reference's scan over the rows of its window -- including the
// reference's upper bound, which stops one row short of the last occupied
// row when the window reaches it -- and the kept points are compacted in
// sorted order.
#include <algorithm>
#include <type_traits>

#include <cub/cub.cuh>

#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

// Order-preserving key of a value: 32-bit for element types of 4 bytes or
// less (halving the shared-memory scans), 64-bit otherwise.
template <typename T>
using KeyOf = typename std::conditional<(sizeof(T) <= 4), uint32_t, unsigned long long>::type;

template <typename T>
__device__ __forceinline__ KeyOf<T> okey(T v) {
  if constexpr (std::is_same<T, float>::value) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  } else if constexpr (sizeof(T) <= 4) {
    if constexpr (std::is_signed<T>::value) return (uint32_t)(int32_t)v ^ 0x80000000u;
    else return (uint32_t)v;
  } else if constexpr (std::is_signed<T>::value) {
    return (unsigned long long)(long long)v ^ 0x8000000000000000ull;
  } else {
    return (unsigned long long)v;
  }
}

constexpr int kRowThreads = 256;
constexpr int kRowBand = 8;  // rows per block of the row pass

// Row pass: for every pixel, the column of its row window's winner (bx) and
// that winner's key (bk). A block takes 256 columns (+ r halo) of kRowBand
// rows, loads all their keys into shared memory at once, then scans.
template <typename T>
__global__ void __launch_bounds__(kRowThreads) snm_rows_kernel(const T* __restrict__ img, uint32_t W, uint32_t H,
                                                               uint32_t r, uint32_t* __restrict__ bx,
                                                               KeyOf<T>* __restrict__ bk) {
  using K = KeyOf<T>;
  extern __shared__ __align__(16) unsigned char s_raw[];
  K* s_key = reinterpret_cast<K*>(s_raw);  // [kRowBand][kRowThreads + 2r]
  const uint32_t seg = kRowThreads + 2 * r;
  const uint32_t xs = blockIdx.x * kRowThreads;  // first pixel of the segment
  const uint32_t lo = xs > r ? xs - r : 0u;
  const uint32_t hi = (uint32_t)min((unsigned long long)W, (unsigned long long)xs + kRowThreads + r);
  const uint32_t y0 = blockIdx.y * kRowBand;
  const uint32_t nrow = min((uint32_t)kRowBand, H - y0);
  for (uint32_t j = 0; j < nrow; ++j) {
    const T* row = img + (size_t)(y0 + j) * W;
    for (uint32_t c = lo + threadIdx.x; c < hi; c += kRowThreads) s_key[j * seg + c - lo] = okey(row[c]);
  }
  __syncthreads();
  const uint32_t x = xs + threadIdx.x;
  if (x >= W) return;
  const uint32_t a = x > r ? x - r : 0u;
  const uint32_t b = (uint32_t)min((unsigned long long)W - 1, (unsigned long long)x + r);
  for (uint32_t j = 0; j < nrow; ++j) {
    const K* kr = s_key + j * seg - lo;
    uint32_t best = a;
    K bkey = kr[a];
    for (uint32_t c = a + 1; c <= b; ++c) {
      const K k = kr[c];
      if (k > bkey) {  // strictly greater: the smaller column wins among equals
        bkey = k;
        best = c;
      }
    }
    bx[(size_t)(y0 + j) * W + x] = best;
    bk[(size_t)(y0 + j) * W + x] = bkey;
  }
}

// Row pass for windows wider than shared memory holds: the same scan from
// global memory.
template <typename T>
__global__ void __launch_bounds__(kRowThreads) snm_rows_global_kernel(const T* __restrict__ img, uint32_t W,
                                                                      uint32_t H, uint32_t r,
                                                                      uint32_t* __restrict__ bx,
                                                                      KeyOf<T>* __restrict__ bk) {
  using K = KeyOf<T>;
  const uint32_t x = blockIdx.x * kRowThreads + threadIdx.x;
  if (x >= W) return;
  for (uint32_t y = blockIdx.y; y < H; y += gridDim.y) {
    const T* row = img + (size_t)y * W;
    const uint32_t a = x > r ? x - r : 0u;
    const uint32_t b = (uint32_t)min((unsigned long long)W - 1, (unsigned long long)x + r);
    uint32_t best = a;
    K bkey = okey(row[a]);
    for (uint32_t c = a + 1; c <= b; ++c) {
      const K k = okey(row[c]);
      if (k > bkey) {
        bkey = k;
        best = c;
      }
    }
    bx[(size_t)y * W + x] = best;
    bk[(size_t)y * W + x] = bkey;
  }
}

// Column pass: winner of the column window over the row winners; the pixel
// keeps its value iff it is the winner. Ties go to the smaller x, then the
// smaller y (the reference's tuple order (x, y)).
template <typename T>
__global__ void __launch_bounds__(256) snm_cols_kernel(const T* __restrict__ img, uint32_t W, uint32_t H, uint32_t r,
                                                       const uint32_t* __restrict__ bx,
                                                       const KeyOf<T>* __restrict__ bk, T* __restrict__ out) {
  using K = KeyOf<T>;
  const uint32_t x = blockIdx.x * 32 + (threadIdx.x & 31);
  const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (x >= W || y >= H) return;
  const uint32_t a = y > r ? y - r : 0u;
  const uint32_t b = (uint32_t)min((unsigned long long)H - 1, (unsigned long long)y + r);
  uint32_t wx = bx[(size_t)a * W + x], wy = a;
  K wk = bk[(size_t)a * W + x];
  for (uint32_t yy = a + 1; yy <= b; ++yy) {
    const uint32_t cx = bx[(size_t)yy * W + x];
    const K k = bk[(size_t)yy * W + x];
    if (k > wk || (k == wk && cx < wx)) {  // equal x: the earlier row already holds
      wk = k;
      wx = cx;
      wy = yy;
    }
  }
  const T v = img[(size_t)y * W + x];
  out[(size_t)y * W + x] = (wx == x && wy == y) ? v : T(0);
}

// Column pass through a shared-memory tile of 32 columns x 32 output rows and
// r halo rows above and below: every row winner of the tile (its column and
// key, both read coalesced) is staged once, then each thread scans its column
// window in shared memory.
constexpr int kColTile = 32;

template <typename T>
__global__ void __launch_bounds__(256) snm_cols_tile_kernel(const T* __restrict__ img, uint32_t W, uint32_t H,
                                                            uint32_t r, const uint32_t* __restrict__ bx,
                                                            const KeyOf<T>* __restrict__ bk, T* __restrict__ out) {
  using K = KeyOf<T>;
  extern __shared__ __align__(16) unsigned char s_raw[];
  const uint32_t trows = kColTile + 2 * r;
  K* s_wk = reinterpret_cast<K*>(s_raw);                                    // [trows][32] winner keys
  uint32_t* s_wx = reinterpret_cast<uint32_t*>(s_wk + (size_t)trows * 32);  // [trows][32] their columns
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t x = blockIdx.x * 32 + lane;
  const uint32_t y0 = blockIdx.y * kColTile;
  const uint32_t lo = y0 > r ? y0 - r : 0u;
  const uint32_t hi = (uint32_t)min((unsigned long long)H, (unsigned long long)y0 + kColTile + r);
  if (x < W)
    for (uint32_t i = warp; i < hi - lo; i += 8) {
      const size_t at = (size_t)(lo + i) * W + x;
      s_wx[i * 32 + lane] = bx[at];
      s_wk[i * 32 + lane] = bk[at];
    }
  __syncthreads();
  if (x >= W) return;
  for (uint32_t k = 0; k < kColTile / 8; ++k) {
    const uint32_t y = y0 + warp * (kColTile / 8) + k;
    if (y >= H) break;
    const uint32_t a = y > r ? y - r : 0u;
    const uint32_t b = (uint32_t)min((unsigned long long)H - 1, (unsigned long long)y + r);
    uint32_t wx = s_wx[(a - lo) * 32 + lane], wy = a;
    K wk = s_wk[(a - lo) * 32 + lane];
    for (uint32_t yy = a + 1; yy <= b; ++yy) {
      const uint32_t cx = s_wx[(yy - lo) * 32 + lane];
      const K kk = s_wk[(yy - lo) * 32 + lane];
      if (kk > wk || (kk == wk && cx < wx)) {
        wk = kk;
        wx = cx;
        wy = yy;
      }
    }
    out[(size_t)y * W + x] = (wx == x && wy == y) ? img[(size_t)y * W + x] : T(0);
  }
}

// One-pass form for element types of 4 bytes or less and radii up to 16: a
// block owns 128 output columns x 32 output rows, stages the keys of that
// tile and its r halo once, and runs both window passes in shared memory.
// Each element's rank is one 64-bit word, (key << 32) | (0xFFFF - col) << 16 |
// (0xFFFF - row) in tile-local coordinates, so the plain maximum is the
// reference's winner (largest value, then smaller x, then smaller y) and 0
// stands for the clipped-away cells outside the image. Both passes find
// window maxima by van Herk / Gil-Werman: a thread owns k = 2r + 1
// consecutive outputs, keeps the suffix maxima of their first inputs in
// registers and sweeps the prefix maxima of the next k, so each output
// costs two maxima whatever the radius (instead of a scan of 2r + 1).
constexpr uint32_t kFusedTW = 128, kFusedTH = 32, kFusedThreads = 256;

template <uint32_t KMAX, typename In, typename Emit>
__device__ __forceinline__ void vhgw_run(uint32_t k, uint32_t n_in, uint32_t n_out, const uint32_t base,
                                         uint64_t (&h)[KMAX], const In& in, const Emit& emit) {
  // suffix maxima of inputs base .. base + k - 1
  uint64_t run = 0;
#pragma unroll
  for (int t = KMAX - 1; t >= 0; --t)
    if ((uint32_t)t < k) {
      const uint32_t c = base + t;
      const uint64_t v = c < n_in ? in(c) : 0ull;
      run = v > run ? v : run;
      h[t] = run;
    }
  // prefix maxima of inputs base + k .. base + 2k - 2, merged into the outputs
  run = 0;
#pragma unroll
  for (uint32_t t = 0; t < KMAX; ++t)
    if (t < k) {
      const uint32_t o = base + t;
      if (o < n_out) emit(o, h[t] > run ? h[t] : run);
      const uint32_t c = base + k + t;
      const uint64_t v = c < n_in ? in(c) : 0ull;
      run = v > run ? v : run;
    }
}

template <typename T>
__device__ __forceinline__ T from_okey(uint32_t k) {
  if constexpr (std::is_same<T, float>::value) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
  } else if constexpr (std::is_signed<T>::value) {
    return (T)(int32_t)(k ^ 0x80000000u);
  } else {
    return (T)k;
  }
}

template <typename T, uint32_t KMAX>
__global__ void __launch_bounds__(kFusedThreads) snm_fused_kernel(const T* __restrict__ img, uint32_t W, uint32_t H,
                                                                  uint32_t r, T* __restrict__ out) {
  static_assert(sizeof(T) <= 4, "32-bit keys");
  extern __shared__ __align__(16) unsigned char s_raw[];
  const uint32_t k = 2 * r + 1;
  const uint32_t ic = kFusedTW + 2 * r, ir = kFusedTH + 2 * r;
  uint64_t* s_row = reinterpret_cast<uint64_t*>(s_raw);            // [ir][kFusedTW] row-window winners
  uint32_t* s_key = reinterpret_cast<uint32_t*>(s_row + ir * kFusedTW);  // [ir][ic] keys
  const long long x0 = (long long)blockIdx.x * kFusedTW, y0 = (long long)blockIdx.y * kFusedTH;
  const long long gx0 = x0 - r, gy0 = y0 - r;
  // stage the keys; cells outside the image are never read as keys (their
  // rank is 0, decided from the coordinates)
  for (uint32_t idx = threadIdx.x; idx < ir * ic; idx += kFusedThreads) {
    const uint32_t i = idx / ic, c = idx - i * ic;
    const long long gy = gy0 + i, gx = gx0 + c;
    uint32_t key = 0;
    if (gy >= 0 && gy < (long long)H && gx >= 0 && gx < (long long)W) key = okey(img[(size_t)gy * W + gx]);
    s_key[idx] = key;
  }
  __syncthreads();
  // row pass: for tile-local row i and output column o, the winner of input
  // columns o .. o + 2r
  const uint32_t nseg = (kFusedTW + k - 1) / k;
  const long long col_lo = -gx0, col_hi = (long long)W - gx0;  // local columns inside the image
  for (uint32_t task = threadIdx.x; task < ir * nseg; task += kFusedThreads) {
    const uint32_t i = task / nseg, seg = task - i * nseg;
    const long long gy = gy0 + i;
    const bool row_in = gy >= 0 && gy < (long long)H;
    const uint32_t* kr = s_key + i * ic;
    const uint64_t rowbits = 0xFFFFu - i;
    uint64_t h[KMAX];
    vhgw_run<KMAX>(
        k, ic, kFusedTW, seg * k, h,
        [&](uint32_t c) -> uint64_t {
          if (!row_in || (long long)c < col_lo || (long long)c >= col_hi) return 0ull;
          return ((uint64_t)kr[c] << 32) | ((uint64_t)(0xFFFFu - c) << 16) | rowbits;
        },
        [&](uint32_t o, uint64_t v) { s_row[i * kFusedTW + o] = v; });
  }
  __syncthreads();
  // column pass: for output (o, j), the winner of row winners j .. j + 2r of
  // column o; the pixel keeps its value iff it is that winner
  const uint32_t nseg2 = (kFusedTH + k - 1) / k;
  for (uint32_t task = threadIdx.x; task < kFusedTW * nseg2; task += kFusedThreads) {
    const uint32_t o = task % kFusedTW, seg = task / kFusedTW;
    const long long gx = x0 + o;
    if (gx >= (long long)W) continue;
    uint64_t h[KMAX];
    vhgw_run<KMAX>(
        k, ir, kFusedTH, seg * k, h, [&](uint32_t i) -> uint64_t { return s_row[i * kFusedTW + o]; },
        [&](uint32_t j, uint64_t v) {
          const long long gy = y0 + j;
          if (gy >= (long long)H) return;
          const uint32_t own = ((0xFFFFu - (o + r)) << 16) | (0xFFFFu - (j + r));
          out[(size_t)gy * W + gx] = (uint32_t)v == own ? from_okey<T>((uint32_t)(v >> 32)) : T(0);
        });
  }
}

size_t snm_fused_smem(uint32_t r) {
  return (size_t)(kFusedTH + 2 * r) * (kFusedTW * 8 + (kFusedTW + 2 * r) * 4);
}

template <typename T, uint32_t KMAX>
cudaError_t launch_snm_fused(const T* img, uint32_t W, uint32_t H, uint32_t r, T* out, cudaStream_t s) {
  static PerDeviceOnce attr;
  cudaError_t e = attr.run([] {
    return cudaFuncSetAttribute(snm_fused_kernel<T, KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)snm_fused_smem((KMAX - 1) / 2));
  });
  if (e != cudaSuccess) return e;
  const dim3 grid((W + kFusedTW - 1) / kFusedTW, (H + kFusedTH - 1) / kFusedTH);
  snm_fused_kernel<T, KMAX><<<grid, kFusedThreads, snm_fused_smem(r), s>>>(img, W, H, r, out);
  count_launch(kKernelSuppress);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_snm_t(const T* img, uint32_t W, uint32_t H, uint32_t r, T* out, void* scratch, cudaStream_t s) {
  using K = KeyOf<T>;
  if (W == 0 || H == 0) return cudaSuccess;
  // the one-pass form reads neighbouring tiles' pixels, so it needs an output
  // apart from the image; tiles are counted in 16 bits (rows of grid.y)
  if constexpr (sizeof(T) <= 4) {
    const bool apart = (const void*)img != (const void*)out;
    if (apart && r <= 16 && (H + kFusedTH - 1) / kFusedTH <= 65535u) {
      if (r <= 4) return launch_snm_fused<T, 9>(img, W, H, r, out, s);
      if (r <= 8) return launch_snm_fused<T, 17>(img, W, H, r, out, s);
      return launch_snm_fused<T, 33>(img, W, H, r, out, s);
    }
  }
  uint32_t* bx = static_cast<uint32_t*>(scratch);
  K* bk = reinterpret_cast<K*>(static_cast<uint8_t*>(scratch) + align_up((size_t)W * H * 4, 256));
  const size_t band = (size_t)kRowBand * (kRowThreads + 2 * (size_t)r) * sizeof(K);
  const uint32_t bands = (H + kRowBand - 1) / kRowBand;
  if (band <= 48 * 1024 && bands <= 65535u) {
    snm_rows_kernel<T><<<dim3((W + kRowThreads - 1) / kRowThreads, bands), kRowThreads, band, s>>>(img, W, H, r,
                                                                                                   bx, bk);
  } else {
    const dim3 rg((W + kRowThreads - 1) / kRowThreads, H < 65535u ? H : 65535u);
    snm_rows_global_kernel<T><<<rg, kRowThreads, 0, s>>>(img, W, H, r, bx, bk);
  }
  count_launch(kKernelSuppress);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t tile_bytes = ((size_t)kColTile + 2 * (size_t)r) * 32 * (sizeof(K) + 4);
  if (tile_bytes <= 48 * 1024) {
    if ((H + kColTile - 1) / kColTile > 65535u) return cudaErrorInvalidValue;  // images up to 2097120 rows
    snm_cols_tile_kernel<T><<<dim3((W + 31) / 32, (H + kColTile - 1) / kColTile), 256, tile_bytes, s>>>(
        img, W, H, r, bx, bk, out);
  } else {
    if ((H + 7) / 8 > 65535u) return cudaErrorInvalidValue;  // images up to 524280 rows
    snm_cols_kernel<T><<<dim3((W + 31) / 32, (H + 7) / 8), 256, 0, s>>>(img, W, H, r, bx, bk, out);
  }
  count_launch(kKernelSuppress);
  return cudaGetLastError();
}

}  // namespace

size_t suppress_scratch_bytes(int type, uint32_t W, uint32_t H) {
  const size_t key = (type == IPB_ELEM_U64 || type == IPB_ELEM_I64) ? 8 : 4;
  return align_up((size_t)W * H * 4, 256) + (size_t)W * H * key;
}

namespace {

// ---- local_maxima ------------------------------------------------------------

__global__ void lm_keys_kernel(const uint32_t* xs, const uint32_t* ys, uint32_t n, unsigned long long* keys,
                               uint32_t* idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    keys[i] = ((unsigned long long)ys[i] << 32) | xs[i];
    idx[i] = i;
  }
}

// row_start[y] = first sorted position with row >= y, for y = 0 .. height + 1
__global__ void lm_rows_kernel(const unsigned long long* skeys, uint32_t n, uint32_t* row_start, uint32_t rows) {
  const uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= rows) return;
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) / 2;
    if ((uint32_t)(skeys[mid] >> 32) < y) lo = mid + 1;
    else hi = mid;
  }
  row_start[y] = lo;
}

__global__ void lm_flags_kernel(const unsigned long long* skeys, const uint32_t* sidx, const float* scores,
                                uint32_t n, uint32_t radius, uint32_t height, const uint32_t* row_start,
                                uint32_t* flags) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t cy = (uint32_t)(skeys[i] >> 32), cx = (uint32_t)skeys[i];
  const float cs = scores[sidx[i]];
  // u32 arithmetic as in the reference (release builds wrap)
  const uint32_t row_lower = cy > radius ? cy - radius : 0u;
  const uint32_t row_upper = (uint32_t)(cy + radius + 1u) > height ? height : (uint32_t)(cy + radius + 1u);
  uint32_t is_max = 1;
  for (uint32_t y = row_lower; y < row_upper && is_max; ++y)
    for (uint32_t k = row_start[y]; k < row_start[y + 1]; ++k) {
      const uint32_t x = (uint32_t)skeys[k];
      if ((uint32_t)(x + radius) < cx) continue;
      if (x > (uint32_t)(cx + radius)) break;
      const float s = scores[sidx[k]];
      if (s > cs) {
        is_max = 0;
        break;
      }
      if (s < cs) continue;
      if (y < cy || (y == cy && x < cx)) {  // (c.y, c.x) < (cy, cx)
        is_max = 0;
        break;
      }
    }
  flags[i] = is_max;
}

__global__ void lm_compact_kernel(const uint32_t* flags, const uint32_t* pos, const uint32_t* sidx, uint32_t n,
                                  uint32_t* out, uint32_t* count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flags[i]) out[pos[i]] = sidx[i];
  if (i == n - 1) *count = pos[i] + flags[i];
}

}  // namespace

cudaError_t launch_suppress(int type, const void* img, uint32_t W, uint32_t H, uint32_t r, void* out, void* bx,
                            cudaStream_t s) {
  switch (type) {
    case IPB_ELEM_U8: return launch_snm_t(static_cast<const uint8_t*>(img), W, H, r, static_cast<uint8_t*>(out), bx, s);
    case IPB_ELEM_U16:
      return launch_snm_t(static_cast<const uint16_t*>(img), W, H, r, static_cast<uint16_t*>(out), bx, s);
    case IPB_ELEM_U32:
      return launch_snm_t(static_cast<const uint32_t*>(img), W, H, r, static_cast<uint32_t*>(out), bx, s);
    case IPB_ELEM_U64:
      return launch_snm_t(static_cast<const unsigned long long*>(img), W, H, r,
                          static_cast<unsigned long long*>(out), bx, s);
    case IPB_ELEM_I8: return launch_snm_t(static_cast<const int8_t*>(img), W, H, r, static_cast<int8_t*>(out), bx, s);
    case IPB_ELEM_I16:
      return launch_snm_t(static_cast<const int16_t*>(img), W, H, r, static_cast<int16_t*>(out), bx, s);
    case IPB_ELEM_I32:
      return launch_snm_t(static_cast<const int32_t*>(img), W, H, r, static_cast<int32_t*>(out), bx, s);
    case IPB_ELEM_I64:
      return launch_snm_t(static_cast<const long long*>(img), W, H, r, static_cast<long long*>(out), bx, s);
    case IPB_ELEM_F32: return launch_snm_t(static_cast<const float*>(img), W, H, r, static_cast<float*>(out), bx, s);
    default: return cudaErrorInvalidValue;
  }
}

size_t local_maxima_scratch_bytes(uint32_t n, uint32_t max_y) {
  size_t sort_tmp = 0, scan_tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (const unsigned long long*)nullptr,
                                  (unsigned long long*)nullptr, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int)n);
  cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n);
  const size_t per = align_up((size_t)n * 8, 256);
  const size_t per4 = align_up((size_t)n * 4, 256);
  return 2 * per + 5 * per4 + align_up(((size_t)max_y + 2) * 4, 256) + align_up(std::max(sort_tmp, scan_tmp), 256) +
         256;
}

// Inputs on the device; out (n indices) and count on the device.
cudaError_t launch_local_maxima(const uint32_t* xs, const uint32_t* ys, const float* scores, uint32_t n,
                                uint32_t radius, uint32_t max_y, void* scratch, size_t scratch_bytes,
                                uint32_t* out, uint32_t* count, cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
  uint8_t* p = static_cast<uint8_t*>(scratch);
  auto take = [&](size_t bytes) {
    void* q = p;
    p += align_up(bytes, 256);
    return q;
  };
  auto* keys = static_cast<unsigned long long*>(take((size_t)n * 8));
  auto* skeys = static_cast<unsigned long long*>(take((size_t)n * 8));
  auto* idx = static_cast<uint32_t*>(take((size_t)n * 4));
  auto* sidx = static_cast<uint32_t*>(take((size_t)n * 4));
  auto* flags = static_cast<uint32_t*>(take((size_t)n * 4));
  auto* pos = static_cast<uint32_t*>(take((size_t)n * 4));
  take((size_t)n * 4);
  auto* row_start = static_cast<uint32_t*>(take(((size_t)max_y + 2) * 4));
  void* tmp = p;
  size_t tmp_bytes = scratch_bytes - (size_t)(p - static_cast<uint8_t*>(scratch));
  const uint32_t blocks = (n + 255) / 256;
  lm_keys_kernel<<<blocks, 256, 0, s>>>(xs, ys, n, keys, idx);
  count_launch(kKernelSuppress);
  // radix sort is stable: equal (y, x) keep their input order
  cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, skeys, idx, sidx, (int)n, 0, 64, s);
  if (e != cudaSuccess) return e;
  // rows 0 .. max_y + 1 (max_y bounds every y, so row_start covers the
  // height the reference takes from the last sorted point)
  lm_rows_kernel<<<(max_y + 2 + 255) / 256, 256, 0, s>>>(skeys, n, row_start, max_y + 2);
  count_launch(kKernelSuppress);
  // height = the largest y: the last sorted key's row, read on the device
  lm_flags_kernel<<<blocks, 256, 0, s>>>(skeys, sidx, scores, n, radius, max_y, row_start, flags);
  count_launch(kKernelSuppress);
  e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flags, pos, (int)n, s);
  if (e != cudaSuccess) return e;
  lm_compact_kernel<<<blocks, 256, 0, s>>>(flags, pos, sidx, n, out, count);
  count_launch(kKernelSuppress);
  return cudaGetLastError();
}

}  // namespace ipb
