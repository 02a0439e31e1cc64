// tm_shift.cu -- exact unmasked template matching on the 5th-generation
// tensor cores with the image row itself as the MMA's A operand.
//
// Replaces the scalar walk of methods::*::score_at (src/template_matching.rs:
// 219-376) for unmasked matches of one template against one or more images
// whose rows are 16-byte aligned (width a multiple of 16), with
// find_extremes (:479-511) optionally fused into the epilogue.
//
// Formulation. A tile is 2048 output columns (x0 + 16m + s for m = 0..127,
// s = 0..15) by NT = 8 output rows (y0 + j). For every image row
// r = y0 + rho (rho = 0 .. NT + h - 2) and K step kk (32 bytes):
//   A_rho[m][k] = I[r][x0 + 16m + k]                           k < K
//   B_rho[(j, s)][k] = T[rho - j][k - s]   (0 <= k - s < w, 0 <= rho - j < h)
//   D[m][(j, s)] += sum_k A_rho[m][k] * B_rho[(j, s)][k]
// so that D[m][(j, s)] = sum_{dy,dx} I[y0+j+dy][x0+16m+s+dx] T[dy][dx] = X,
// with K = w + 15 rounded up to 32 (the 16 shifts s of each template row
// live in B). A needs no building: in the canonical no-swizzle K-major
// layout a core matrix is eight 16-byte rows, and with 16 bytes between the
// two K halves (LBO) and 128 bytes between 8-row groups (SBO) the descriptor
// of the staged image row at byte 32 kk reads row m at byte 16m + 32 kk --
// the overlapping windows of the row, straight from shared memory. B for
// image row rho is a window of one buffer: the template rows' 16-shift blocks
// (16 rows of K bytes each) stored in decreasing template row, so the blocks
// of j = j_lo .. j_hi (the output rows that image row feeds) are consecutive,
// starting at block h - 1 - (rho - j_lo); the MMA's N is 16 (j_hi - j_lo + 1)
// and its accumulator columns start at 16 j_lo, so no zero rows are issued.
// A first MMA with zero operands (a zeroed buffer read through the same
// overlapping descriptor) clears the tile's accumulator.
//
// Y = sum I^2 over each window (SumOfSquaredErrors and the normalised
// methods) comes from a window-sum map built beforehand by two separable
// passes (vsum_kernel, hsum_kernel; u32: w h 255^2 < 2^32 for the template
// sizes taken here), once per image of a launch; TSS and the template's
// 16-shift blocks from shift_prep_kernel, once per launch.
//
// Pipeline: one loader warp copies each image row segment (2048 + K bytes,
// less at the image's right edge) with 16-byte cp.async copies into a ring of
// shared-memory slots, two loader warps taking the rows in turn with several
// in flight each; one warp issues the MMAs of a
// row once its slot is full and commits the slot back; eight epilogue warps
// (two per tensor-memory lane quadrant, four tile rows each) drain each
// finished tile from one of two accumulator buffers of 128 columns while the
// MMAs of the next tile run. The template blocks arrive by bulk copies once
// per CTA.
// Every wait is bounded (a budget per tile, so the global timer is read once
// per tile on the fast path, not once per row); a wait that runs out records
// the launch's tag in the error word and the CTA leaves its loops, drains its
// MMAs and frees its tensor memory.
#include <algorithm>

#include "tm_common.cuh"
#include "tm_internal.h"
#include "tm_sm100.cuh"

namespace ipb {
namespace {

using namespace sm100;

constexpr uint32_t kLanes = 128;            // M: column groups of 16
constexpr uint32_t kTileW = kLanes * 16;    // output columns per tile
constexpr uint32_t kNT = 8;                 // output rows per tile (N = 128)
constexpr uint32_t kAccCols = kNT * 16;     // accumulator columns per buffer
constexpr uint32_t kStages = 16;            // image-row slots at most (8 at least)
constexpr uint32_t kEpiWarps = 8, kMmaWarp = 8, kLoadWarp = 9, kLoadWarps = 2;
constexpr uint32_t kThreads = (kLoadWarp + kLoadWarps) * 32;
constexpr int kRowsInFlight = 3;  // per loader warp; kLoadWarps x kRowsInFlight < the slots
// the zero operands of the clearing MMA: A (128 rows) and B (kAccCols rows),
// both read through the overlapping descriptor, 16 bytes per row
constexpr uint32_t kZeroBytes = 16 * (kAccCols - 1) + 32 + 16;
constexpr uint32_t kHeader = 1024;  // barriers and flags
constexpr uint32_t kZeroRegion = (kZeroBytes + 127) / 128 * 128;
constexpr uint32_t kStageFloats = 2 * (512 + 32);  // per epilogue warp: Y and scores, 1 pad per 16
constexpr uint32_t kRingOff = kHeader + kZeroRegion + kEpiWarps * kStageFloats * 4;
constexpr uint32_t kMaxK = 160;

struct ShiftProblem {
  const uint8_t* img;     // pitch = W bytes, 16-byte aligned rows
  const uint32_t* ymap;   // Wo x Ho window sums of I^2, or null (CrossCorrelation)
  float* out;             // Wo x Ho, or null (extremes only)
  unsigned long long* ext;  // {min key, max key} or null
  uint32_t W, H, Wo, Ho;
  uint32_t tiles_x, tile_begin;
  int method, precision;
};

constexpr uint32_t kMaxProblems = 8;
static_assert(kMaxProblems == kShiftMaxProblems, "problems per launch");

struct ShiftLaunch {
  ShiftProblem p[kMaxProblems];
  uint32_t nprobs, tiles;
  const uint8_t* blocks;  // h blocks of 16 K bytes, then TSS (u32)
  uint32_t h, K, rowbytes, stages;
  uint32_t ring_off, b_off;
  unsigned int* err;
  unsigned int tag;
  unsigned long long wait_ns;
};

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t problem_of(const ShiftLaunch& L, uint32_t tile) {
  uint32_t p = 0;
  while (p + 1 < L.nprobs && tile >= L.p[p + 1].tile_begin) ++p;
  return p;
}

struct TileCoord {
  uint32_t p, x0, y0, nrows;
};
__device__ __forceinline__ TileCoord tile_coord(const ShiftLaunch& L, uint32_t tile) {
  TileCoord t;
  t.p = problem_of(L, tile);
  const ShiftProblem& q = L.p[t.p];
  const uint32_t lt = tile - q.tile_begin;
  t.x0 = (lt % q.tiles_x) * kTileW;
  t.y0 = (lt / q.tiles_x) * kNT;
  t.nrows = min(kNT + L.h - 1, q.H - t.y0);
  return t;
}

// Epilogue of part of a tile for one warp (tensor-memory lanes 32w .. 32w +
// 31, i.e. output columns x0 + 512w .. x0 + 512w + 511; tile rows j0 .. j1 -
// 1). Row by row: the warp's 16 x 32 accumulators come out of tensor memory
// with one load, the window
// sums Y of the row segment go through the warp's staging area (coalesced
// global loads, then each lane's 16 columns), the scores are finished in
// registers, folded into the extremes and written back through the staging
// area as coalesced rows. The staging area pads every 16 floats by one, so
// both the lane-major and the row-major accesses are free of bank conflicts.
struct EpiTile {
  const ShiftProblem& pr;
  const TileCoord& t;
  uint32_t taddr;  // lane quadrant and accumulator buffer
  float* stage;
  uint32_t warp, lane, tss;  // warp: the lane quadrant
  uint32_t j0, j1;           // the warp's tile rows
};

__device__ __forceinline__ uint32_t stage_at(uint32_t i) { return i + (i >> 4); }

template <int kMethod, bool kFp64>
__device__ __forceinline__ void epi_tile(const EpiTile& e) {
  constexpr bool kNeedY = kMethod != kCcorr;
  const ShiftProblem& pr = e.pr;
  const uint32_t xw = e.t.x0 + 512 * e.warp;  // the warp's first column
  if (xw >= pr.Wo) return;
  const uint32_t ncols = min(512u, pr.Wo - xw), nrow = min(e.j1, pr.Ho - e.t.y0);
  if (e.j0 >= nrow) return;
  uint32_t* ystage = reinterpret_cast<uint32_t*>(e.stage);
  float* ostage = e.stage + 512 + 32;
  unsigned long long kmin = ~0ull, kmax = 0ull;
  // the next row's accumulators and window sums are in flight while a row is
  // finished
  uint32_t xn[16], yn[16];
  tmem_ld16(e.taddr + 16 * e.j0, xn);
  size_t row = (size_t)(e.t.y0 + e.j0) * pr.Wo + xw;
  if constexpr (kNeedY) {
#pragma unroll
    for (uint32_t q = 0; q < 16; ++q) {
      const uint32_t i = e.lane + 32 * q;
      yn[q] = i < ncols ? pr.ymap[row + i] : 0u;
    }
  }
  const uint32_t c0 = 16 * e.lane;
  for (uint32_t j = e.j0; j < nrow; ++j, row += pr.Wo) {
    if constexpr (kNeedY) {
#pragma unroll
      for (uint32_t q = 0; q < 16; ++q) ystage[stage_at(e.lane + 32 * q)] = yn[q];
    }
    tmem_wait_ld();
    uint32_t xv[16];
#pragma unroll
    for (uint32_t s = 0; s < 16; ++s) xv[s] = xn[s];
    if (j + 1 < nrow) {
      tmem_ld16(e.taddr + 16 * (j + 1), xn);
      if constexpr (kNeedY) {
#pragma unroll
        for (uint32_t q = 0; q < 16; ++q) {
          const uint32_t i = e.lane + 32 * q;
          yn[q] = i < ncols ? pr.ymap[row + pr.Wo + i] : 0u;
        }
      }
    }
    __syncwarp();
    uint32_t mn = 0xFFFFFFFFu, jmn = 0, mx = 0u, jmx = 0;
#pragma unroll
    for (uint32_t s = 0; s < 16; ++s) {
      const uint32_t yw = kNeedY ? ystage[stage_at(c0 + s)] : 0u;
      const uint32_t bits = __float_as_uint(
          finish_score32(kMethod, kFp64 ? IPB_PRECISION_EXACT_FP64 : IPB_PRECISION_EXACT_F32, xv[s], yw, e.tss));
      xv[s] = bits;
      if (c0 + s < ncols) {
        if (bits < mn) {
          mn = bits;
          jmn = s;
        }
        if (bits > mx) {
          mx = bits;
          jmx = s;
        }
      }
    }
    if (pr.ext && c0 < ncols) {
      const uint32_t lin = (uint32_t)row + c0;
      kmin = min(kmin, ((unsigned long long)(mn | 0x80000000u) << 32) | (lin + jmn));
      kmax = max(kmax, ((unsigned long long)(mx | 0x80000000u) << 32) | (0xFFFFFFFFu - (lin + jmx)));
    }
    if (pr.out) {
#pragma unroll
      for (uint32_t s = 0; s < 16; ++s) ostage[stage_at(c0 + s)] = __uint_as_float(xv[s]);
      __syncwarp();
#pragma unroll 4
      for (uint32_t i = e.lane; i < ncols; i += 32) pr.out[row + i] = ostage[stage_at(i)];
    }
    __syncwarp();
  }
  if (pr.ext) {
    for (int o = 16; o > 0; o >>= 1) {
      kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
      kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (e.lane == 0 && kmin != ~0ull) {
      atomicMin(pr.ext, kmin);
      atomicMax(pr.ext + 1, kmax);
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1) shift_match_kernel(const __grid_constant__ ShiftLaunch L) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);       // [kStages]
  uint64_t* empty = full + kStages;                          // [kStages]
  uint64_t* acc_full = empty + kStages;                      // [2]
  uint64_t* acc_empty = acc_full + 2;                        // [2]
  uint64_t* drain = acc_empty + 2;                           // [1]
  uint64_t* bbar = drain + 1;                                // [1] template blocks landed
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bbar + 1);
  uint32_t* s_flag = s_tmem + 1;                             // a wait ran out
  uint8_t* zero_a = smem + kHeader;
  uint8_t* ring = smem + L.ring_off;
  uint8_t* bbuf = smem + L.b_off;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t h = L.h, K = L.K, blk = 16 * K;

  // ---- set-up: barriers, tensor memory, the zero operand, the template's
  // 16-shift blocks and TSS
  if (tid == 0) {
    for (uint32_t i = 0; i < kStages; ++i) {
      mbar_init(full + i, 1);
      mbar_init(empty + i, 1);
    }
    for (uint32_t i = 0; i < 2; ++i) {
      mbar_init(acc_full + i, 1);
      mbar_init(acc_empty + i, kEpiWarps);
    }
    mbar_init(drain, 1);
    mbar_init(bbar, 1);
    *s_flag = 0;
    mbar_init_fence();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(s_tmem, 2 * kAccCols);
    tmem_relinquish();
  }
  for (uint32_t i = tid; i < kZeroBytes / 4; i += kThreads) reinterpret_cast<uint32_t*>(zero_a)[i] = 0u;
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // the template's 16-shift blocks, prepared once per template in global
  // memory (shift_prep_kernel), arrive by bulk copies; only the MMA warp
  // waits for them
  const uint32_t bbytes = h * blk;
  if (tid == 0) {
    mbar_arrive_expect_tx(bbar, bbytes);
    for (uint32_t o = 0; o < bbytes; o += 32768u)
      bulk_g2s(smem_u32(bbuf + o), L.blocks + o, min(32768u, bbytes - o), bbar);
  }
  const uint32_t tss = *reinterpret_cast<const uint32_t*>(L.blocks + bbytes);
  const uint32_t tbase = *s_tmem;
  const uint32_t G = gridDim.x;

  if (warp >= kLoadWarp) {
    // ---- loaders: kLoadWarps warps take the image rows in turn (row q to
    // warp q % kLoadWarps); a row is 16-byte cp.async copies spread over the
    // warp, committed as one group. A warp keeps kRowsInFlight of its rows in
    // flight and hands the oldest to the MMA warp: every lane waits for its
    // copies of it (wait_group), makes them visible to the tensor core's
    // proxy, and after the warp has synchronised one lane arrives on the row.
    // Slots and phases advance by increments (no divisions per row).
    const uint32_t lw = warp - kLoadWarp;
    uint32_t q = 0, mine = 0, handed = 0;  // rows seen; this warp's rows issued and handed
    uint32_t slot = 0, u = 0;              // slot of row q and its use count
    uint32_t hq[kRowsInFlight + 1];        // this warp's rows not yet handed (ring)
    for (uint32_t tile = blockIdx.x; tile < L.tiles && !*reinterpret_cast<volatile uint32_t*>(s_flag);
         tile += G) {
      const TileCoord t = tile_coord(L, tile);
      const ShiftProblem& pr = L.p[t.p];
      const uint32_t chunks = min(L.rowbytes, pr.W - t.x0) / 16;  // W is a multiple of 16
      // one budget per tile: the global timer is read once here, not per row
      const unsigned long long deadline = global_ns() + L.wait_ns;
      bool ok = true;
      for (uint32_t rho = 0; rho < t.nrows; ++rho) {
        if (q % kLoadWarps == lw) {
          if (u > 0 && !mbar_wait(empty + slot, (u - 1) & 1, deadline)) {
            if (lane == 0) {
              atomicMax(L.err, L.tag);
              *s_flag = 1;
            }
            ok = false;
            break;
          }
          // bytes of the slot past the image row keep whatever they held: an
          // output column x < Wo reads image bytes x .. x + w - 1 <= W - 1
          // only, every other byte of its K window meets a zero of B, and the
          // columns x >= Wo that do read them are never stored
          const uint32_t dst = smem_u32(ring + slot * L.rowbytes);
          const uint8_t* src = pr.img + (size_t)(t.y0 + rho) * pr.W + t.x0;
          for (uint32_t c = lane; c < chunks; c += 32) cp_async16(dst + 16 * c, src + 16 * c);
          cp_async_commit();
          hq[mine % (kRowsInFlight + 1)] = slot;
          ++mine;
          if (mine - handed > kRowsInFlight) {
            cp_async_wait_group<kRowsInFlight>();
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(full + hq[handed % (kRowsInFlight + 1)]);
            ++handed;
          }
        }
        ++q;
        if (++slot == L.stages) {
          slot = 0;
          ++u;
        }
      }
      if (!ok) break;
    }
    cp_async_wait_all();
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0)
      for (; handed < mine; ++handed) mbar_arrive(full + hq[handed % (kRowsInFlight + 1)]);
  } else if (warp == kMmaWarp) {
    // ---- MMA issue
    uint32_t q = 0, it = 0;
    bool ok = true;
    const uint32_t zdesc_a = smem_u32(zero_a), bb = smem_u32(bbuf), rb = smem_u32(ring);
    ok = mbar_wait(bbar, 0, global_ns() + L.wait_ns);
    for (uint32_t tile = blockIdx.x; tile < L.tiles && ok; tile += G, ++it) {
      const TileCoord t = tile_coord(L, tile);
      const uint32_t buf = it & 1, v = it >> 1;
      // one budget per tile: the global timer is read once here, not per row
      const unsigned long long deadline = global_ns() + L.wait_ns;
      if (v > 0 && !mbar_wait(acc_empty + buf, (v - 1) & 1, deadline)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t dcol = tbase + buf * kAccCols;
      mma_i8_ss_warp(dcol, smem_desc_noswizzle(zdesc_a, 16, 128), smem_desc_noswizzle(zdesc_a, 16, 128),
                     idesc_u8u8_s32(kLanes, kAccCols), 0u);
      for (uint32_t rho = 0; rho < t.nrows; ++rho, ++q) {
        const uint32_t slot = q % L.stages, u = q / L.stages;
        if (!mbar_wait(full + slot, u & 1, deadline)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t jlo = rho + 1 > h ? rho + 1 - h : 0u, jhi = min(kNT - 1, rho);
        const uint32_t n = 16 * (jhi - jlo + 1);
        const uint32_t idesc = idesc_u8u8_s32(kLanes, n);
        const uint32_t b0 = bb + (h - 1 - (rho - jlo)) * blk, a0 = rb + slot * L.rowbytes;
        for (uint32_t kk = 0; kk < K / 32; ++kk)
          mma_i8_ss_warp(dcol + 16 * jlo, smem_desc_noswizzle(a0 + 32 * kk, 16, 128),
                         smem_desc_noswizzle(b0 + 256 * kk, 128, 8 * K), idesc, 1u);
        mma_commit_warp(empty + slot);
      }
      if (!ok) break;
      mma_commit_warp(acc_full + buf);
    }
    if (!ok && lane == 0) {
      atomicMax(L.err, L.tag);
      *s_flag = 1;
    }
    // drain: every MMA issued has completed before tensor memory is freed
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kDefaultWaitNs) && lane == 0) atomicMax(L.err, L.tag);
  } else {
    // ---- epilogue: warp w drains tensor-memory lanes 32 (w % 4) .. + 31,
    // tile rows 4 (w / 4) .. + 3
    float* stage = reinterpret_cast<float*>(smem + kHeader + kZeroRegion) + warp * kStageFloats;
    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < L.tiles; tile += G, ++it) {
      const TileCoord t = tile_coord(L, tile);
      const ShiftProblem& pr = L.p[t.p];
      const uint32_t buf = it & 1, v = it >> 1;
      if (!mbar_wait_sleep(acc_full + buf, v & 1, global_ns() + L.wait_ns)) {
        if (lane == 0) {
          atomicMax(L.err, L.tag);
          *s_flag = 1;
        }
        break;
      }
      tc_fence_after();
      const uint32_t quad = warp & 3, half = warp >> 2;
      EpiTile e{pr, t, tbase + ((32 * quad) << 16) + buf * kAccCols, stage, quad, lane, tss,
                half * (kNT / 2), half * (kNT / 2) + kNT / 2};
      const bool fp64 = pr.precision == IPB_PRECISION_EXACT_FP64;
      switch (pr.method) {
        case kSse: fp64 ? epi_tile<kSse, true>(e) : epi_tile<kSse, false>(e); break;
        case kSseNorm: fp64 ? epi_tile<kSseNorm, true>(e) : epi_tile<kSseNorm, false>(e); break;
        case kCcorr: epi_tile<kCcorr, true>(e); break;
        default: fp64 ? epi_tile<kCcorrNorm, true>(e) : epi_tile<kCcorrNorm, false>(e); break;
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty + buf);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tbase, 2 * kAccCols);
}

// The template side, once per template: block b = h - 1 - dy holds rows
// s = 0..15 of K bytes, byte k = T[dy][k - s] (0 outside the template), in
// the canonical no-swizzle K-major layout (s / 8) * 8K + (k / 16) * 128 +
// (s % 8) * 16 + k % 16, built a 32-bit word per thread; then TSS = sum T^2
// (the last block of the grid).
__global__ void __launch_bounds__(256) shift_prep_kernel(const uint8_t* __restrict__ tpl, uint32_t w, uint32_t h,
                                                         uint32_t K, uint8_t* __restrict__ blocks) {
  const uint32_t words = h * 16 * (K / 4);
  if (blockIdx.x == gridDim.x - 1) {
    __shared__ uint32_t red[8];
    uint32_t tss = 0;
    for (uint32_t i = threadIdx.x; i < w * h; i += 256) {
      const uint32_t v = tpl[i];
      tss += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) tss += __shfl_xor_sync(0xffffffffu, tss, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tss;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t total = 0;
      for (int i = 0; i < 8; ++i) total += red[i];
      *reinterpret_cast<uint32_t*>(blocks + (size_t)h * 16 * K) = total;
    }
    return;
  }
  const uint32_t i = blockIdx.x * 256 + threadIdx.x;
  if (i >= words) return;
  const uint32_t kw = K / 4, b = i / (16 * kw), rem = i - b * 16 * kw;
  const uint32_t s = rem / kw, k = (rem - s * kw) * 4;
  const uint8_t* trow = tpl + (size_t)(h - 1 - b) * w;
  uint32_t word = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int c = (int)(k + e) - (int)s;
    const uint32_t v = (c >= 0 && c < (int)w) ? trow[c] : 0u;
    word |= v << (8 * e);
  }
  *reinterpret_cast<uint32_t*>(blocks + (size_t)b * 16 * K + (s >> 3) * 8 * K + (k >> 4) * 128 + (s & 7) * 16 +
                               (k & 15)) = word;
}

// Y[y][x] = sum over the w x h window at (x, y) of I^2 (u32), for the Wo x Ho
// output positions, in two separable passes through a scratch map V:
//  * vsum_kernel: V[y][x] = sum_{dy < h} I[y + dy][x]^2 for every image
//    column x and output row y: a thread owns four columns (one aligned word
//    per row) and 32 output rows, slides its four sums down them (one word
//    in, one out per row) and stores them as one 16-byte word per row;
//  * hsum_kernel: a block takes one output row, stages V's row in shared
//    memory (coalesced) and each thread slides a w-wide sum along a run of 16
//    output columns.
constexpr uint32_t kVRows = 32;

__device__ __forceinline__ void add_squares(uint32_t v, uint32_t (&a)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t b = (v >> (8 * k)) & 255u;
    a[k] += b * b;
  }
}
__device__ __forceinline__ void sub_squares(uint32_t v, uint32_t (&a)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t b = (v >> (8 * k)) & 255u;
    a[k] -= b * b;
  }
}

__global__ void __launch_bounds__(256) vsum_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t H,
                                                   uint32_t h, uint32_t* __restrict__ vmap) {
  const uint32_t Ho = H - h + 1, words = W / 4;  // W is a multiple of 16
  const uint32_t wc = blockIdx.x * 256 + threadIdx.x, y0 = blockIdx.y * kVRows;
  if (wc >= words) return;
  const uint32_t rows = min(kVRows, Ho - y0);
  const uint32_t* src = reinterpret_cast<const uint32_t*>(img) + wc;
  uint32_t a[4] = {0u, 0u, 0u, 0u};
  for (uint32_t dy = 0; dy < h; ++dy) add_squares(src[(size_t)(y0 + dy) * words], a);
  uint4* dst = reinterpret_cast<uint4*>(vmap + (size_t)y0 * W) + wc;
  dst[0] = make_uint4(a[0], a[1], a[2], a[3]);
  for (uint32_t j = 1; j < rows; ++j) {
    add_squares(src[(size_t)(y0 + j + h - 1) * words], a);
    sub_squares(src[(size_t)(y0 + j - 1) * words], a);
    dst[(size_t)j * words] = make_uint4(a[0], a[1], a[2], a[3]);
  }
}

__global__ void __launch_bounds__(256) hsum_kernel(const uint32_t* __restrict__ vmap, uint32_t W, uint32_t w,
                                                   uint32_t* __restrict__ ymap) {
  extern __shared__ uint32_t s_v[];  // one V row, one pad word per 16
  const uint32_t Wo = W - w + 1, y = blockIdx.x;
  const uint32_t* vr = vmap + (size_t)y * W;
  for (uint32_t i = threadIdx.x; i < W; i += 256) s_v[i + (i >> 4)] = vr[i];
  __syncthreads();
  uint32_t* yr = ymap + (size_t)y * Wo;
  for (uint32_t x = 16 * threadIdx.x; x < Wo; x += 16 * 256) {
    uint32_t acc = 0;
    for (uint32_t dx = 0; dx < w; ++dx) {
      const uint32_t i = x + dx;
      acc += s_v[i + (i >> 4)];
    }
    yr[x] = acc;
    const uint32_t n = min(16u, Wo - x);
    for (uint32_t k = 1; k < n; ++k) {
      const uint32_t ia = x + k + w - 1, ib = x + k - 1;
      acc += s_v[ia + (ia >> 4)] - s_v[ib + (ib >> 4)];
      yr[x + k] = acc;
    }
  }
}

// image-row slots: 16, fewer (down to 8) where the template blocks leave
// less room
uint32_t shift_stages(uint32_t w, uint32_t h) {
  const uint32_t K = (w + 15 + 31) & ~31u;
  const size_t fixed = kRingOff + (size_t)h * 16 * K, rowbytes = kTileW + K;
  for (uint32_t st = kStages; st > 8; --st)
    if (fixed + st * rowbytes <= 227u * 1024u) return st;
  return 8;
}

size_t shift_smem_bytes(uint32_t w, uint32_t h) {
  const uint32_t K = (w + 15 + 31) & ~31u;
  const size_t rowbytes = kTileW + K;
  // at least 120 KB: one CTA per SM, so two CTAs never wait on each other's
  // tensor memory
  return std::max<size_t>(kRingOff + shift_stages(w, h) * rowbytes + (size_t)h * 16 * K, 120u * 1024u);
}

size_t blocks_bytes(uint32_t w, uint32_t h) {
  const uint32_t K = (w + 15 + 31) & ~31u;
  return (size_t)h * 16 * K + 16;
}

// the window sums and, ahead of them, the column sums they are made from
size_t ymap_bytes(const MatchArgs& a) {
  return align_up((size_t)(a.W - a.w + 1) * (a.H - a.h + 1) * 4, 256) + align_up((size_t)a.W * (a.H - a.h + 1) * 4, 256);
}

// problems [0, n) that need the window sums of an image: the first problem on
// each distinct image (same pointer and size) owns its map
bool owns_ymap(const MatchArgs* a, uint32_t i) {
  if (a[i].method == IPB_CROSS_CORRELATION) return false;
  for (uint32_t k = 0; k < i; ++k)
    if (a[k].method != IPB_CROSS_CORRELATION && a[k].img == a[i].img && a[k].W == a[i].W && a[k].H == a[i].H)
      return false;
  return true;
}

}  // namespace

bool shift_supported(const MatchArgs& a) {
  if (a.mask || a.precision == IPB_PRECISION_REFERENCE_F32) return false;
  if (a.w == 0 || a.h == 0 || a.w > a.W || a.h > a.H) return false;
  if ((a.W & 15u) || (reinterpret_cast<uintptr_t>(a.img) & 15u)) return false;
  if ((uint64_t)a.w * a.h > 33025u) return false;
  const uint32_t K = (a.w + 15 + 31) & ~31u;
  if (K > kMaxK || (size_t)a.W * 4 * 17 / 16 + 64 > 200u * 1024u) return false;
  return shift_smem_bytes(a.w, a.h) <= 227u * 1024u;
}

bool shift_preferred(const MatchArgs& a) {
  const int path = kernel_path();
  if (path == 3) return shift_supported(a);
  return false;
}

size_t shift_multi_scratch_bytes(const MatchArgs* a, uint32_t n) {
  size_t bytes = align_up(blocks_bytes(a[0].w, a[0].h), 256);
  for (uint32_t i = 0; i < n; ++i)
    if (owns_ymap(a, i)) bytes += ymap_bytes(a[i]);
  return bytes;
}

size_t shift_scratch_bytes(const MatchArgs& a) { return shift_multi_scratch_bytes(&a, 1); }

cudaError_t launch_shift_multi(const MatchArgs* a, unsigned long long* const* ext, uint32_t n, void* scratch,
                               unsigned int* err, unsigned int tag, cudaStream_t stream, KernelTimer* timer) {
  if (n == 0 || n > kMaxProblems) return cudaErrorInvalidValue;
  for (uint32_t i = 1; i < n; ++i)  // one template side per launch
    if (a[i].tpl != a[0].tpl || a[i].w != a[0].w || a[i].h != a[0].h) return cudaErrorInvalidValue;
  static PerDeviceOnce attr;
  cudaError_t e = attr.run([] {
    cudaError_t r = cudaFuncSetAttribute(shift_match_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(hsum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  });
  if (e != cudaSuccess) return e;
  const uint32_t w = a[0].w, h = a[0].h;
  const uint32_t K = (w + 15 + 31) & ~31u;
  uint8_t* sc = static_cast<uint8_t*>(scratch);
  uint8_t* blocks = sc;
  size_t off = align_up(blocks_bytes(w, h), 256);
  const uint32_t words = h * 16 * (K / 4);
  shift_prep_kernel<<<(words + 255) / 256 + 1, 256, 0, stream>>>(a[0].tpl, w, h, K, blocks);
  count_launch(kKernelPrep);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  ShiftLaunch L{};
  uint32_t tiles = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t Wo = a[i].W - w + 1, Ho = a[i].H - h + 1;
    ShiftProblem& p = L.p[i];
    if (owns_ymap(a, i)) {
      uint32_t* vmap = reinterpret_cast<uint32_t*>(sc + off);
      p.ymap = reinterpret_cast<uint32_t*>(sc + off + align_up((size_t)a[i].W * Ho * 4, 256));
      off += ymap_bytes(a[i]);
      const dim3 vg((a[i].W / 4 + 255) / 256, (Ho + kVRows - 1) / kVRows);
      if (vg.y > 65535u || Ho > 2147483647u) return cudaErrorInvalidValue;
      vsum_kernel<<<vg, 256, 0, stream>>>(a[i].img, a[i].W, a[i].H, h, vmap);
      hsum_kernel<<<Ho, 256, ((size_t)a[i].W + a[i].W / 16 + 1) * 4, stream>>>(vmap, a[i].W, w,
                                                                             const_cast<uint32_t*>(p.ymap));
      count_launch(kKernelWindowSq);
      count_launch(kKernelWindowSq);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else if (a[i].method != IPB_CROSS_CORRELATION) {
      for (uint32_t k = 0; k < i; ++k)
        if (L.p[k].ymap && a[k].img == a[i].img && a[k].W == a[i].W && a[k].H == a[i].H) p.ymap = L.p[k].ymap;
    }
    p.img = a[i].img;
    p.out = a[i].out;
    p.ext = ext ? ext[i] : nullptr;
    p.W = a[i].W;
    p.H = a[i].H;
    p.Wo = Wo;
    p.Ho = Ho;
    p.tiles_x = (Wo + kTileW - 1) / kTileW;
    p.tile_begin = tiles;
    p.method = a[i].method;
    p.precision = a[i].precision;
    tiles += p.tiles_x * ((Ho + kNT - 1) / kNT);
  }
  L.nprobs = n;
  L.tiles = tiles;
  L.blocks = blocks;
  L.h = h;
  L.K = K;
  L.rowbytes = kTileW + K;
  L.ring_off = kRingOff;
  L.stages = shift_stages(w, h);
  L.b_off = kRingOff + L.stages * L.rowbytes;
  L.err = err;
  L.tag = tag;
  L.wait_ns = pipeline_wait_ns();
  const uint32_t grid = std::min<uint32_t>(L.tiles, (uint32_t)device_sm_count());
  timer_begin(timer, kKernelRows, stream);
  shift_match_kernel<<<grid, kThreads, shift_smem_bytes(w, h), stream>>>(L);
  timer_end(timer, stream);
  count_launch(kKernelRows);
  return cudaGetLastError();
}

cudaError_t launch_shift(const MatchArgs& a, void* scratch, unsigned long long* ext, unsigned int* err,
                         unsigned int tag) {
  unsigned long long* const exts[1] = {ext};
  return launch_shift_multi(&a, exts, 1, scratch, err, tag, a.stream, a.timer);
}

}  // namespace ipb
