// tm_head_tc.cu -- the proposal network's heatmap on the 5th-generation
// tensor cores, reduced on the fly to the maximum of each 8 x 8 cell.
//
// z_t(p) = alpha * sum_o F(p + o) . G_t(o), o in {(0,0), (0,1), (1,0), (1,1)}
// (F: the image's 32-channel features, row-chunked bf16; G_t: template t's
// 2 x 2 x 32 embedding). A tile is one feature row y and 128 positions
// x0 .. x0 + 127 (M = 128 = tensor-memory lanes) against a group of up to 64
// templates (N); K = 4 offsets x 32 channels = 8 MMAs of K = 16. The A
// operand of offset (oy, ox) is the staged feature row y + oy started ox
// pixels (16 * ox bytes) later, the same no-swizzle K-major layout as the
// convolutions. A CTA walks the 8 rows of one cell row of a 128-position
// segment: a loader warp stages rows into a ring, the MMA warp issues each
// row's 8 MMAs into one of two accumulators, and four epilogue warps keep, per
// template, the running maximum over the cell's rows in registers; after the
// 8th row the 8 lanes of each cell fold their maxima with shuffles. The cell
// key is (order key of the logit << 32) | ~position, so ties go to the smaller
// position -- the same keys as the reduction it replaces.
#include "imageproc_b200.h"
#include "tm_internal.h"
#include "tm_learned.cuh"
#include "tm_sm100.cuh"

namespace ipb {
namespace learned {
namespace {

using namespace sm100;

constexpr int kHSeg = 128;                     // positions per tile
constexpr int kHRowPx = 136;                   // staged pixels per row (129 used)
constexpr int kHChunkBytes = kHRowPx * 16;     // 2176 B
constexpr int kHRowBytes = kChunks * kHChunkBytes;
constexpr int kHRing = 3;                      // staged feature rows
constexpr int kHCell = 8;                      // cell side
constexpr int kHN = 64;                        // templates per CTA
constexpr int kHThreads = 192;                 // warp 0 MMA, warp 1 loader, warps 2..5 epilogue
constexpr uint32_t kHTmemCols = 128;           // two accumulators of 64 columns

struct HeadLayout {
  static constexpr uint32_t g = 0;                                  // [o][chunk][64 templates] x 16 B
  static constexpr uint32_t ring = 4 * kChunks * kHN * 16;          // 16384
  static constexpr uint32_t bars = ring + kHRing * kHRowBytes;
  static constexpr uint32_t misc = bars + 16 * 8;
  // at least 48 KB, so at most four CTAs share an SM's 512 tensor-memory columns
  static constexpr uint32_t total = misc + 16 > 48u * 1024u ? misc + 16 : 48u * 1024u;
};

__host__ __device__ constexpr uint32_t idesc_bf16_f32_h(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss_h(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void cp_async16_z(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ uint32_t okey_h(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

struct HeadArgs {
  const uint4* F;        // Hs x 4 x Ws units
  const uint16_t* gb;    // [4 offsets][T][32] bf16
  uint32_t Hs, Ws, T;
  unsigned long long* cells;  // [T][Cy][Cx]
  unsigned long long wait_ns;
  uint32_t stall;
  unsigned int* err;
  unsigned int tag;
};

__global__ void __launch_bounds__(kHThreads) head_tc_kernel(const HeadArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* row_full = reinterpret_cast<uint64_t*>(smem + HeadLayout::bars);
  uint64_t* row_empty = row_full + kHRing;
  uint64_t* acc_full = row_empty + kHRing;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + HeadLayout::misc);
  volatile uint32_t* s_err = s_tmem + 1;

  const uint32_t x0 = blockIdx.x * kHSeg, cy = blockIdx.y, t0 = blockIdx.z * kHN;
  const uint32_t y0 = cy * kHCell;
  const uint32_t nrows = min((uint32_t)kHCell, a.Hs - y0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // embeddings: [o][chunk][template] 16-byte units (K-major B), zero past T
  for (uint32_t i = threadIdx.x; i < 4u * kHN * kChunks; i += kHThreads) {
    const uint32_t c = i & 3u, row = i >> 2, o = row / kHN, tl = row % kHN;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (t0 + tl < a.T) v = reinterpret_cast<const uint4*>(a.gb)[((size_t)o * a.T + t0 + tl) * kChunks + c];
    reinterpret_cast<uint4*>(smem + HeadLayout::g)[(o * kChunks + c) * kHN + tl] = v;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kHRing; ++s) {
      mbar_init(&row_full[s], 1);
      mbar_init(&row_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(drain, 1);
    *s_err = 0;
    mbar_init_fence();
  }
  fence_proxy_async_smem();
  if (warp == 0) {
    tmem_alloc(s_tmem, kHTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long deadline = global_ns() + a.wait_ns;
  const uint32_t ring0 = smem_u32(smem + HeadLayout::ring);
  const uint32_t g0 = smem_u32(smem + HeadLayout::g);

  if (warp == 1) {
    // loader: feature rows y0 .. y0 + nrows (one past the cell: offset oy = 1)
    for (uint32_t i = 0; i <= nrows; ++i) {
      const uint32_t s = i % kHRing, u = i / kHRing;
      if (u > 0 && !mbar_wait(&row_empty[s], (u - 1) & 1u, deadline)) {
        *s_err = 1;
        break;
      }
      const uint32_t y = y0 + i;
      const bool row_ok = y < a.Hs;
      const uint32_t dst0 = ring0 + s * kHRowBytes;
      for (uint32_t j = lane; j < (uint32_t)(kChunks * (kHSeg + 1)); j += 32) {
        const uint32_t c = j / (kHSeg + 1), px = j % (kHSeg + 1);
        const uint32_t x = x0 + px;
        const bool ok = row_ok && x < a.Ws;
        const uint4* src = ok ? a.F + (((size_t)y * kChunks + c) * a.Ws + x) : a.F;
        cp_async16_z(dst0 + c * kHChunkBytes + px * 16, src, ok ? 16u : 0u);
      }
      asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&row_full[s]);
    }
  } else if (warp == 0) {
    constexpr uint32_t idesc = idesc_bf16_f32_h(kHSeg, kHN);
    const bool leader = elect_one();
    if (a.stall && !__all_sync(0xffffffffu, mbar_wait(drain, 0, deadline))) *s_err = 1;
    for (uint32_t k = 0; k < nrows && !*s_err; ++k) {
      bool ok = mbar_wait(&row_full[k % kHRing], (k / kHRing) & 1u, deadline) &&
                mbar_wait(&row_full[(k + 1) % kHRing], ((k + 1) / kHRing) & 1u, deadline);
      const uint32_t b = k & 1u, v = k >> 1;
      if (ok && v > 0) ok = mbar_wait(&acc_empty[b], (v - 1) & 1u, deadline);
      if (!__all_sync(0xffffffffu, ok)) {
        *s_err = 1;
        break;
      }
      tc_fence_after();
      if (leader) {
        const uint32_t d = tmem + b * kHN;
#pragma unroll
        for (uint32_t o = 0; o < 4; ++o) {
          const uint32_t oy = o >> 1, ox = o & 1;
          const uint32_t arow = ring0 + ((k + oy) % kHRing) * kHRowBytes + ox * 16;
#pragma unroll
          for (uint32_t js = 0; js < 2; ++js) {
            const uint64_t ad = smem_desc_noswizzle(arow + 2 * js * kHChunkBytes, kHChunkBytes, 128);
            const uint64_t bd = smem_desc_noswizzle(g0 + (o * kChunks + 2 * js) * kHN * 16, kHN * 16, 128);
            mma_bf16_ss_h(d, ad, bd, idesc, (o | js) != 0);
          }
        }
        mma_commit(&acc_full[b]);
        mma_commit(&row_empty[k % kHRing]);  // row k is not read again
      }
      __syncwarp();
    }
  } else {
    // epilogue: lane quadrant q, position x = x0 + 32 q + lane
    const uint32_t q = warp & 3;
    const uint32_t x = x0 + 32 * q + lane;
    float best[kHN];
    uint32_t rows_of[kHN / 8];  // 4 bits per template: the row (0..7) of its maximum
#pragma unroll
    for (int t = 0; t < kHN; ++t) best[t] = -INFINITY;
#pragma unroll
    for (int t = 0; t < kHN / 8; ++t) rows_of[t] = 0u;
    bool ok = true;
    for (uint32_t k = 0; k < nrows; ++k) {
      const uint32_t b = k & 1u, v = k >> 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], v & 1u, deadline))) {
        *s_err = 1;
        ok = false;
        break;
      }
      tc_fence_after();
      uint32_t r[32];
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        tmem_ld32(tmem_addr(tmem, 32 * q, b * kHN + 32 * half), r);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int t = 32 * half + j;
          const float z = kAlpha * __uint_as_float(r[j]);
          if (z > best[t]) {  // strict: the earlier row keeps a tie
            best[t] = z;
            rows_of[t >> 3] = (rows_of[t >> 3] & ~(0xFu << (4 * (t & 7)))) | (k << (4 * (t & 7)));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    if (ok) {
      // fold the 8 lanes (positions) of each cell: value first, then the
      // smaller position (row first, then column)
      const uint32_t Cx = (a.Ws + kHCell - 1) / kHCell;
      const uint32_t cx = x / kHCell;
#pragma unroll
      for (int t = 0; t < kHN; ++t) {
        const uint32_t rw = (rows_of[t >> 3] >> (4 * (t & 7))) & 0xFu;
        const bool valid = x < a.Ws;
        unsigned long long key =
            valid ? ((unsigned long long)okey_h(best[t]) << 32) | (0xFFFFFFFFu - ((y0 + rw) * a.Ws + x)) : 0ull;
#pragma unroll
        for (int d = 1; d < kHCell; d <<= 1) {
          const unsigned long long o2 = __shfl_xor_sync(0xffffffffu, key, d);
          key = o2 > key ? o2 : key;
        }
        if ((lane & (kHCell - 1)) == 0 && valid && t0 + t < a.T)
          a.cells[((size_t)(t0 + t) * gridDim.y + cy) * Cx + cx] = key;
      }
    }
  }

  __syncthreads();
  if (warp == 0) {
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kDefaultWaitNs)) *s_err = 1;
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kHTmemCols);
  }
  if (threadIdx.x == 0 && *s_err && a.err) atomicMax(a.err, a.tag);
}

}  // namespace

cudaError_t launch_head_tc(const uint4* F, uint32_t Hs, uint32_t Ws, const uint16_t* gb, uint32_t T,
                           unsigned long long* cells, unsigned int* err, unsigned int tag, cudaStream_t s) {
  if (T == 0 || Hs == 0 || Ws == 0) return cudaSuccess;
  static PerDeviceOnce attr;
  cudaError_t e = attr.run([] {
    return cudaFuncSetAttribute(head_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HeadLayout::total);
  });
  if (e != cudaSuccess) return e;
  const dim3 grid((Ws + kHSeg - 1) / kHSeg, (Hs + kHCell - 1) / kHCell, (T + kHN - 1) / kHN);
  HeadArgs args{F, gb, Hs, Ws, T, cells, pipeline_wait_ns(), pipeline_stall() ? 1u : 0u, err, tag};
  head_tc_kernel<<<grid, kHThreads, HeadLayout::total, s>>>(args);
  count_launch(kKernelPropose);
  return cudaGetLastError();
}

}  // namespace learned
}  // namespace ipb
