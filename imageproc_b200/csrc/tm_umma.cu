// tm_umma.cu -- exact template matching on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, unsigned u8 x u8 -> s32, accumulators in tensor memory).
//
// Replaces the scalar walk of methods::*::score_at (src/template_matching.rs:
// 219-376) for unmasked and binary-masked matches with templates up to
// 256 x 128 pixels (128 x 128 masked), for one problem or a batch of many
// (image, template) pairs of uneven sizes in one persistent launch, with
// find_extremes (:479-511) optionally fused into the epilogue.
//
// Formulation. A CTA owns a tile of 128 output columns (x0 + c(m) for
// tensor-memory lane m, c = lane_column below, a permutation of 0..127) by NT
// output rows (y0 + n, n = tensor-memory column). For each image row r of the
// tile (r = 0 .. NT + h - 2, image row y0 + r) and each correlation c, into
// accumulator a(c) (writing x0 + m for x0 + c(m)):
//   A_r[m][k] = P_c[y0 + r][x0 + m + k]          (a Hankel row per lane)
//   B_r[n][k] = Q_c[r - n][k]                     (0 <= r - n < h, else 0)
//   D_a(c)[m][n] += sum_k A_r[m][k] * B_r[n][k]
// so that after all rows D_a[m][n] = sum over c with a(c) = a of
// sum_{dy,dx} P_c[y0+n+dy][x0+m+dx] Q_c[dy][dx].
//   unmasked:     c = 0: P = I, Q = T,                      a = 0  -> X
//   binary mask:  c = 0: P = I, Q = T*m,                    a = 0  -> X
//                 c = 1: P = I^2 mod 255,       Q = m,      a = 1  \ Y
//                 c = 2: P = floor(I^2 / 255),  Q = 255*m,  a = 1  /
// Both parts of I^2 = 255 floor(I^2/255) + I^2 mod 255 lie in 0..255, and
// 255*m is a u8 for a binary mask, so the two u8 x u8 correlations sum to
// Y = sum I^2 m in one accumulator, exactly: every partial sum is at most
// 65025 * 16384 < 2^31 for the masked template sizes taken here. Masked
// CrossCorrelation needs X alone (the reference's masked score is
// sum I T m^2, src/template_matching.rs:336-351): its problems skip the
// I^2 planes and correlations 1 and 2.
// B_r is a window of one buffer Z_c (Q_c with its rows reversed and 16 zero
// rows on each side) stored in the canonical no-swizzle K-major layout, whose
// rows are 16 bytes apart: moving from r to r+1 moves B's start address by
// -16 bytes. Only the 16-aligned band of n where B_r is non-zero is issued.
//
// A_r goes straight into tensor memory: sixteen builder warps (four per
// tensor-memory lane quadrant) read each lane's window of the staged image row
// as aligned 16-byte chunks, form its K bytes with byte_perm and store them
// with tcgen05.st; the MMA reads A from
// tensor memory and only B from shared memory. Unmasked, the same words give
// the lane's row sum of squares with dp4a, from which the epilogue slides the
// window sum Y = sum I^2 over h rows, so no integral image is needed. The
// kernel builds Z and the template constant TSS from the raw template (and
// mask) whenever a CTA moves to a tile of another problem.
//
// Pipeline: image tiles are double-buffered in shared memory and loaded with
// cp.async while the previous tile is computed. Builders fill 2 stages of RPS
// A rows (two large stages beat three smaller ones in the tensor memory left
// beside the accumulators: each stage hand-off costs a tcgen05.wait::st and two
// mbarrier round trips); one warp runs the MMA issue loop on warp-uniform values and one
// elected lane issues the MMAs of a stage once it is full, then commits it
// back to the builders; after the tile's last stage it commits the
// accumulators to the epilogue (the builder warps), which reads them with
// tcgen05.ld, writes the scores and folds them into the problem's extremes.
// Every wait is bounded (2 s); a wait that runs out records the launch's tag
// in the error word and the CTA leaves its loop, drains its MMAs and frees its
// tensor memory.
#include <algorithm>
#include <tuple>
#include <vector>

#include "tm_common.cuh"
#include "tm_internal.h"
#include "tm_sm100.cuh"

namespace ipb {
namespace {

using namespace sm100;

constexpr int kM = 128;
constexpr int kBuilderWarps = 16;
constexpr int kSubs = kBuilderWarps / 4;  // builder warps per tensor-memory lane quadrant
constexpr int kBuilders = kBuilderWarps * 32;
constexpr int kThreads = kBuilders + 32;
constexpr int kWarps = kThreads / 32;
constexpr int kStages = 2;  // A-row stages in tensor memory
constexpr uint32_t kMaxRps = 16;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned long long kWaitNs = kDefaultWaitNs;  // the final drain's budget
constexpr uint32_t kBandTable = 1024;          // per-row MMA band table (uint4 per image row)
constexpr uint32_t kMaxTileRows = 256;         // NT + h - 1 <= 128 + 128 - 1
constexpr uint32_t kSmemHeader = kBandTable + kMaxTileRows * 16;
constexpr uint32_t kMinSmem = 120 * 1024;  // keeps residency at one CTA per SM

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// first problem of the set that owns a global tile, advancing monotonically
// from the set starting at `pi`
__device__ __forceinline__ uint32_t find_problem(const UmmaLaunch& L, const UmmaProblem* P, uint32_t pi,
                                                 uint32_t tile) {
  for (;;) {
    const uint32_t nx = pi + max(P[pi].set_n, 1u);
    if (nx >= L.nprobs || tile < P[nx].tile_begin) return pi;
    pi = nx;
  }
}

// Template side cached in shared memory per set member slot: the Z buffers
// and TSS stay valid while the slot's template, mask and shape are unchanged
// (consecutive tiles of one set; sets that repeat a template).
struct ZKey {
  const uint8_t* tpl;
  const uint8_t* mask;
  uint32_t w, h, kmma, pad;
};
// shared-memory header below the band table: barriers and flags (0..255),
// TSS partial sums per member and warp, TSS per member, the members' keys
static_assert(256 + kMaxSet * kWarps * 8 + 64 + kMaxSet * sizeof(ZKey) <= kBandTable, "kernel header");

// Stage image rows [y0, y0 + nrows) x columns [x0, x0 + imgp) of plane 0 for
// the problem's local tile, zero past the right edge. Asynchronous unless the
// image rows are not 4-byte aligned.
__device__ void issue_tile_load(const UmmaLaunch& L, const UmmaProblem q, uint8_t* dst_plane, uint32_t lt) {
  const uint32_t x0 = (lt % q.tiles_x) * kM;
  const uint32_t y0 = (lt / q.tiles_x) * L.NT;
  const uint32_t nrows = min(q.rows_max, q.H - y0);
  const uint8_t* src = q.img + (size_t)y0 * q.W;
  if (q.load_mode == 2) {
    const uint32_t chunks = L.imgp / 16;
    for (uint32_t idx = threadIdx.x; idx < nrows * chunks; idx += kThreads) {
      const uint32_t r = idx / chunks, c = (idx % chunks) * 16, gx = x0 + c;
      const uint32_t avail = gx < q.W ? min(16u, q.W - gx) : 0u;
      const uint8_t* g = src + (size_t)r * q.W + (avail ? gx : 0u);
      cp_async16(smem_u32(dst_plane + r * L.imgp + c), g, avail);
    }
  } else if (q.load_mode == 1) {
    const uint32_t words = L.imgp / 4;
    for (uint32_t idx = threadIdx.x; idx < nrows * words; idx += kThreads) {
      const uint32_t r = idx / words, c = (idx % words) * 4, gx = x0 + c;
      const uint32_t avail = gx < q.W ? min(4u, q.W - gx) : 0u;
      const uint8_t* g = src + (size_t)r * q.W + (avail ? gx : 0u);
      cp_async4(smem_u32(dst_plane + r * L.imgp + c), g, avail);
    }
  } else {
    const uint32_t words = L.imgp / 4;
    for (uint32_t idx = threadIdx.x; idx < nrows * words; idx += kThreads) {
      const uint32_t r = idx / words, c = (idx % words) * 4, gx = x0 + c;
      const uint8_t* row = src + (size_t)r * q.W;
      uint32_t v = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (gx + k < q.W) v |= (uint32_t)__ldg(row + gx + k) << (8 * k);
      *reinterpret_cast<uint32_t*>(dst_plane + r * L.imgp + c) = v;
    }
  }
  cp_async_commit();
}

// Output column (offset in the tile) of tensor-memory lane m = 32 q + l:
// 16 (l / 4) + 4 q + (l % 4). Each lane quadrant q takes the columns whose
// word offset within their 16-byte chunk is q, so a builder warp reads its
// lanes' windows with aligned 16-byte loads and one compile-time word
// offset; the four quadrants cover the tile's 128 columns once.
__device__ __forceinline__ uint32_t lane_column(uint32_t m) {
  return 16u * ((m & 31u) >> 2) + 4u * (m >> 5) + (m & 3u);
}

// Builds one A row (one plane) for lane l of lane quadrant Q into tensor
// memory: the lane's window starts at byte 16 (l / 4) + 4 Q + (l % 4) of the
// staged row, read as 16-byte chunks from chunk l / 4 on (the last byte read
// is 128 + 4 KS, inside the row pitch). Returns the lane's row sum of
// squares over the template width when kRowSums.
template <int KS, bool kRowSums, int Q>
__device__ __forceinline__ uint32_t build_row(const uint8_t* plane_row, uint32_t l, uint32_t w,
                                              uint32_t taddr) {
  const uint4* cp = reinterpret_cast<const uint4*>(plane_row) + (l >> 2);
  const uint32_t sel = 0x3210u + (l & 3u) * 0x1111u;
  uint32_t rs = 0;
  // words per tensor-memory store: 16 for rows of 16 words; 8 otherwise, which
  // keeps the wider rows within the 96 registers a thread has
  constexpr int CH = KS == 16 ? 16 : 8;
  const uint32_t wq = w >> 2;
  const uint32_t tail = (w & 3u) ? ((1u << (8u * (w & 3u))) - 1u) : 0u;
  uint4 cur = cp[0];
  // the 64-word rows run their eight groups as a loop (registers)
#pragma unroll(KS == 64 ? 1 : KS / CH)
  for (int c0 = 0; c0 < KS; c0 += CH) {
    // four words of A per chunk, from the chunk and the next one
    uint32_t a[CH];
#pragma unroll
    for (int j = 0; j < CH / 4; ++j) {
      const uint4 nxt = cp[c0 / 4 + j + 1];
      const uint32_t w8[8] = {cur.x, cur.y, cur.z, cur.w, nxt.x, nxt.y, nxt.z, nxt.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) a[4 * j + i] = __byte_perm(w8[Q + i], w8[Q + i + 1], sel);
      cur = nxt;
    }
    if constexpr (kRowSums) {
      if (c0 + CH <= (int)wq) {
        uint32_t r4[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < CH; ++k) r4[k & 3] = __dp4a(a[k], a[k], r4[k & 3]);
        rs += (r4[0] + r4[1]) + (r4[2] + r4[3]);
      } else if (c0 <= (int)wq) {
#pragma unroll
        for (int k = 0; k < CH; ++k) {
          const uint32_t idx = c0 + k;
          const uint32_t v = a[k] & (idx < wq ? 0xFFFFFFFFu : (idx == wq ? tail : 0u));
          rs = __dp4a(v, v, rs);
        }
      }
    }
    if constexpr (CH == 16) tmem_st16(taddr + c0, a);
    else tmem_st8(taddr + c0, a);
  }
  return rs;
}

// One builder warp's share of a pipeline stage's A rows [r0, r_end): rows
// r_first, r_first + kSubs, ... unmasked, with the lanes' row sums of
// squares into s_rs[r][m]; with a mask the stage's (row, plane) builds are
// dealt out over the quadrant's kSubs warps in turn, so that stages of few
// image rows (sets) keep every builder warp busy.
struct StageRows {
  const uint8_t* img_buf;
  uint32_t r_first, r_end, r0, tcol0, a_row_cols, imgp, plane_bytes, lane, m, w, tmem, sub;
  uint32_t* s_rs;
  bool need_y;
};

template <int KS, bool MASKED, int Q>
__device__ __forceinline__ void build_stage_rows(const StageRows& sr) {
  if constexpr (MASKED) {
    const uint32_t npl = sr.need_y ? 3u : 1u;
    const uint32_t items = (sr.r_end - sr.r0) * npl;
    for (uint32_t t = sr.sub; t < items; t += kSubs) {
      const uint32_t i = t / npl, pl = t % npl;
      build_row<KS, false, Q>(sr.img_buf + (sr.r0 + i) * sr.imgp + pl * sr.plane_bytes, sr.lane, sr.w,
                              tmem_addr(sr.tmem, Q * 32, sr.tcol0 + i * sr.a_row_cols + pl * KS));
    }
  } else {
    for (uint32_t r = sr.r_first; r < sr.r_end; r += kSubs)
      sr.s_rs[r * kM + sr.m] = build_row<KS, true, Q>(sr.img_buf + r * sr.imgp, sr.lane, sr.w,
                                                      tmem_addr(sr.tmem, Q * 32, sr.tcol0 + (r - sr.r0) * sr.a_row_cols));
  }
}

// A builder warp's share of a tile's epilogue: columns [c_begin, c_begin +
// ncols) of the accumulators for its 32 lanes (output columns).
struct UmmaEpi {
  const UmmaProblem* q;
  uint32_t tmem, xcol, ycol;  // tensor memory; the member's X and (masked) the set's Y accumulator columns
  uint32_t lane_base, c_begin, ncols, NT, nrows, m, x, y0, tss, lane;
  const uint32_t* s_rs;  // unmasked: row sums of squares of the tile's image rows
  uint32_t Y;            // unmasked: window sum of the first column (row c_begin)
};

// Scores with the method and precision fixed at compile time, so the
// kEpiCols scores of each tensor-memory load are straight-line code (eight:
// the accumulator, Y and its two sliding inputs stay within the registers
// the 544-thread block leaves each thread).
constexpr int kEpiCols = 8;
template <bool MASKED, int kMethod, int kPrec, bool kExt>
__device__ __forceinline__ void umma_epilogue(const UmmaEpi& e) {
  const UmmaProblem& q = *e.q;
  uint32_t Y = e.Y;
  unsigned long long kmin = ~0ull, kmax = 0ull;
  for (uint32_t n0 = e.c_begin; n0 < e.c_begin + e.ncols; n0 += kEpiCols) {
    uint32_t vx[kEpiCols];
    tmem_ld8(tmem_addr(e.tmem, e.lane_base, e.xcol + n0), vx);
    uint32_t yv[kEpiCols];
    if constexpr (MASKED && kMethod == kCcorr) {
#pragma unroll
      for (int k = 0; k < kEpiCols; ++k) yv[k] = 0u;  // not computed: CrossCorrelation is X alone
    } else if constexpr (MASKED) {
      tmem_ld8(tmem_addr(e.tmem, e.lane_base, e.ycol + n0), yv);
    } else {
      // window sums of the chunk: loads first, then the sliding chain
      uint32_t add[kEpiCols], subv[kEpiCols];
#pragma unroll
      for (int k = 0; k < kEpiCols; ++k) {
        const uint32_t ra = n0 + k + q.h, rb = n0 + k;
        add[k] = ra < e.nrows ? e.s_rs[ra * kM + e.m] : 0u;
        subv[k] = rb < e.nrows ? e.s_rs[rb * kM + e.m] : 0u;
      }
#pragma unroll
      for (int k = 0; k < kEpiCols; ++k) {
        yv[k] = Y;
        Y += add[k];
        Y -= subv[k];
      }
    }
    tmem_wait_ld();
    // scores are never negative, so their f32 bits order like the values;
    // the lane's positions are rows of one column in index order, so the
    // strict comparisons keep each extreme's first occurrence in the chunk
    const uint32_t y_first = e.y0 + n0;
    const int nv = e.x < q.Wo ? (y_first < q.Ho ? (int)min((uint32_t)kEpiCols, q.Ho - y_first) : 0) : 0;
    uint32_t mn = 0xFFFFFFFFu, jmn = 0, mx = 0u, jmx = 0;
    float* orow = q.out ? q.out + (size_t)y_first * q.Wo + e.x : nullptr;  // null: extremes only
#pragma unroll
    for (int k = 0; k < kEpiCols; ++k) {
      const uint32_t bk = __float_as_uint(finish_score32(kMethod, kPrec, vx[k], yv[k], e.tss));
      if (k < nv) {
        if (orow) orow[(size_t)k * q.Wo] = __uint_as_float(bk);
        if constexpr (kExt) {
          if (bk < mn) {
            mn = bk;
            jmn = k;
          }
          if (bk > mx) {
            mx = bk;
            jmx = k;
          }
        }
      }
    }
    if constexpr (kExt) {
      if (nv > 0) {
        const uint32_t lin0 = y_first * q.Wo + e.x;
        kmin = min(kmin, ((unsigned long long)(mn | 0x80000000u) << 32) | (lin0 + jmn * q.Wo));
        kmax = max(kmax, ((unsigned long long)(mx | 0x80000000u) << 32) | (0xFFFFFFFFu - (lin0 + jmx * q.Wo)));
      }
    }
  }
  if constexpr (kExt) {
    // first occurrence wins: min key = (smallest value, smallest index);
    // max key = (largest value, smallest index) via the complemented index
    for (int o = 16; o > 0; o >>= 1) {
      kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
      kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (e.lane == 0 && kmin != ~0ull) {
      atomicMin(q.ext, kmin);
      atomicMax(q.ext + 1, kmax);
    }
  }
}

template <bool MASKED, int kMethod>
__device__ __forceinline__ void umma_epilogue_m(const UmmaEpi& e, bool fp64, bool ext) {
  if constexpr (!method_is_norm(kMethod)) fp64 = true;  // precision only affects the normalisation
  if (fp64) {
    if (ext) umma_epilogue<MASKED, kMethod, IPB_PRECISION_EXACT_FP64, true>(e);
    else umma_epilogue<MASKED, kMethod, IPB_PRECISION_EXACT_FP64, false>(e);
  } else {
    if (ext) umma_epilogue<MASKED, kMethod, IPB_PRECISION_EXACT_F32, true>(e);
    else umma_epilogue<MASKED, kMethod, IPB_PRECISION_EXACT_F32, false>(e);
  }
}

template <bool MASKED>
__device__ __forceinline__ void umma_epilogue_dispatch(const UmmaEpi& e, int method, bool fp64, bool ext) {
  switch (method) {
    case kSse: umma_epilogue_m<MASKED, kSse>(e, fp64, ext); break;
    case kSseNorm: umma_epilogue_m<MASKED, kSseNorm>(e, fp64, ext); break;
    case kCcorr: umma_epilogue_m<MASKED, kCcorr>(e, fp64, ext); break;
    default: umma_epilogue_m<MASKED, kCcorrNorm>(e, fp64, ext); break;
  }
}

// The MMAs of one pipeline stage, issued by the elected lane: for each of
// the stage's cnt image rows (reading four band entries {n0, idesc, first Z
// row} ahead of their MMAs; the reads run at most three entries past the
// tile's last row, still inside shared memory since the Z buffers follow the
// table, and are unused), each of the set's NS members multiplies the row's
// A (tensor memory) by its own template side (Z, shared memory) into its own
// accumulators over the row's band of output rows.
struct StageIssue {
  const uint4* band;
  uint32_t r0, cnt, a_stage, a_row_cols, dlo, dhi, zslot16, zoff1, kstride, ksteps, tmem, NT, ycol, ymask;
};

template <int NS, int KS, bool MASKED>
__device__ __forceinline__ void issue_stage(const StageIssue& si) {
  constexpr int NCORR = MASKED ? 3 : 1;  // correlations, one per plane
  for (uint32_t i0 = 0; i0 < si.cnt; i0 += 4) {
    uint4 bd[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) bd[j] = si.band[si.r0 + i0 + j];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (i0 + j < si.cnt) {
        const uint32_t n0 = bd[j].x, idesc = bd[j].y;
        const uint32_t zrow = si.dlo + bd[j].z;
        const uint32_t a = si.a_stage + (i0 + j) * si.a_row_cols;
        // X: each member's own template side into its own accumulator
#pragma unroll
        for (int p = 0; p < NS; ++p) {
          const uint32_t zo = zrow + p * si.zslot16;
#pragma unroll
          for (uint32_t kk = 0; kk < (uint32_t)(KS / 8); ++kk) {
            if (kk < si.ksteps)
              mma_i8_ts(si.tmem + p * si.NT + n0, a + kk * 8, ((uint64_t)si.dhi << 32) | (zo + kk * si.kstride),
                        idesc, 1u);
          }
        }
        // Y = sum I^2 m: both parts of I^2 against the members' common mask
        // (the first member's m and 255 m), once per set, unless every
        // member is CrossCorrelation (X alone)
        if (MASKED && si.ymask) {
#pragma unroll
          for (int c = 1; c < NCORR; ++c) {
            const uint32_t zo = zrow + c * si.zoff1;
#pragma unroll
            for (uint32_t kk = 0; kk < (uint32_t)(KS / 8); ++kk) {
              if (kk < si.ksteps)
                mma_i8_ts(si.tmem + si.ycol + n0, a + c * KS + kk * 8,
                          ((uint64_t)si.dhi << 32) | (zo + kk * si.kstride), idesc, 1u);
            }
          }
        }
      }
    }
  }
}

// SETS: launches whose plan holds sets of two or more problems; the instance
// for problems alone compiles the member loops away.
template <int KS, bool MASKED, bool SETS>
__global__ void __launch_bounds__(kThreads, 1) umma_match_kernel(const __grid_constant__ UmmaLaunch L) {
  constexpr int NPL = MASKED ? 3 : 1;    // staged image planes: I (, I^2 mod 255, floor(I^2 / 255))
  constexpr int NZ = MASKED ? 3 : 1;     // reversed-template buffers, one per correlation
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  uint64_t* dfull = empty + kStages;
  uint64_t* drain = dfull + 1;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + 128);
  volatile int* s_err = reinterpret_cast<volatile int*>(smem + 132);
  volatile uint32_t* s_next = reinterpret_cast<volatile uint32_t*>(smem + 136);  // tile after the current one
  // [kMaxSet][kWarps] partial sums of TSS, per member slot: TSS, Z keys
  unsigned long long* s_part = reinterpret_cast<unsigned long long*>(smem + 256);
  uint32_t* s_tss = reinterpret_cast<uint32_t*>(smem + 256 + kMaxSet * kWarps * 8);
  ZKey* s_zkey = reinterpret_cast<ZKey*>(smem + 256 + kMaxSet * kWarps * 8 + 64);
  uint8_t* zbuf = smem + L.z_off;
  uint8_t* s_img = smem + L.img_off;
  uint32_t* s_rs = reinterpret_cast<uint32_t*>(smem + L.rs_off);
  const UmmaProblem* P = L.nprobs <= kInlineProblems ? L.inl : L.probs;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool mma_warp = warp == kBuilderWarps;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], kBuilderWarps);  // one arrive per builder warp
      mbar_init(&empty[s], 1);
    }
    mbar_init(dfull, 1);
    mbar_init(drain, 1);
    *s_err = 0;
    for (uint32_t p = 0; p < kMaxSet; ++p) s_zkey[p] = ZKey{nullptr, nullptr, 0u, 0u, 0u, 0u};
    mbar_init_fence();
  }
  if (mma_warp) {
    tmem_alloc(s_tmem, kTmemCols);
    tmem_relinquish();
  }
  uint32_t pi = 0;
  // first tile's rows start streaming in while the template side is prepared
  if (blockIdx.x < L.tiles) {
    pi = find_problem(L, P, 0, blockIdx.x);
    issue_tile_load(L, P[pi], s_img, blockIdx.x - P[pi].tile_begin);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  // accumulators: X of member p at column p NT; masked, the set's Y (its
  // members share the image and the mask, so Y = sum I^2 m is theirs in
  // common) after the members' X; then the A stages
  const uint32_t ycol = (SETS ? L.set_max : 1u) * L.NT;
  const uint32_t a_col0 = ycol + (MASKED ? L.NT : 0u);
  const uint32_t a_row_cols = NPL * KS;

  uint32_t g = 0;            // pipeline stage fills so far (same count in builders and the MMA warp)
  uint32_t tcount = 0;       // tiles finished by this CTA
  bool ok = true;

  for (uint32_t tile = blockIdx.x, next = 0; tile < L.tiles; tile = next, ++tcount) {
    __syncthreads();
    if (*s_err) break;
    // the tile after this one: drawn from the launch's counter when it
    // schedules dynamically (a CTA that starts late, behind another launch,
    // takes fewer tiles), else a fixed grid stride. Claims rise monotonically.
    if (threadIdx.x == 0) *s_next = L.sched ? gridDim.x + atomicAdd(L.sched, 1u) : tile + gridDim.x;
    pi = find_problem(L, P, pi, tile);
    // a register copy: the tcgen05/cp.async asm statements clobber memory,
    // which would otherwise force every use to reload the field
    const UmmaProblem q = P[pi];
    const uint32_t lt = tile - q.tile_begin;
    const uint32_t buf = L.nbuf == 2 ? (tcount & 1u) : 0u;
    uint8_t* img_buf = s_img + buf * NPL * L.plane_bytes;
    if (L.nbuf == 1 && tcount > 0) issue_tile_load(L, q, img_buf, lt);
    const uint32_t x0 = (lt % q.tiles_x) * kM;
    const uint32_t y0 = (lt / q.tiles_x) * L.NT;
    const uint32_t nrows = min(q.rows_max, q.H - y0);
    const uint32_t zplane = (q.kmma / 16) * q.zrows * 16;
    const uint32_t zslot = NZ * zplane;  // template-side bytes per set member
    const uint32_t nset = SETS ? max(q.set_n, 1u) : 1u;
    // members whose template side is not cached in their slot; the members
    // share the image, the template size and therefore the band table
    uint32_t zbits = 0;
    for (uint32_t p = 0; p < nset; ++p) {
      const UmmaProblem& mp = P[pi + p];
      const ZKey k = s_zkey[p];
      if (mp.tpl != k.tpl || mp.mask != k.mask || mp.w != k.w || mp.h != k.h || mp.kmma != k.kmma)
        zbits |= 1u << p;
    }
    if (zbits) {
      // Z buffers of every member to rebuild, in one pass over all of them:
      // K-chunk-major, chunk c holds rows j = 0..zrows-1 of 16 bytes, row
      // j = template row h-1-(j-16) for 16 <= j < h+16, else zero.
      //   unmasked: Z_0 from T;  binary mask: Z_0 from T*m, Z_1 from m, Z_2 from 255*m
      const uint32_t nchunks = q.kmma / 16, per = NZ * nchunks * q.zrows;
      for (uint32_t idx = threadIdx.x; idx < nset * per; idx += kThreads) {
        const uint32_t p = idx / per;
        if (!((zbits >> p) & 1u)) continue;
        const uint8_t* tp = P[pi + p].tpl;
        const uint8_t* mk = P[pi + p].mask;
        const uint32_t zp = (idx % per) / (nchunks * q.zrows);
        const uint32_t rem = idx % (nchunks * q.zrows);
        const uint32_t c = rem / q.zrows, j = rem % q.zrows;
        uint32_t wd[4] = {0u, 0u, 0u, 0u};
        if (j >= 16 && j < q.h + 16) {
          const size_t row = (size_t)(q.h - 1 - (j - 16)) * q.w;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const uint32_t dx = 16 * c + k;
            if (dx < q.w) {
              uint32_t v;
              if constexpr (MASKED) {
                const uint32_t mv = __ldg(mk + row + dx);
                v = zp == 0 ? (uint32_t)__ldg(tp + row + dx) * mv : (zp == 1 ? mv : 255u * mv);
              } else {
                v = __ldg(tp + row + dx);
              }
              wd[k >> 2] |= (v & 0xFFu) << (8 * (k & 3));
            }
          }
        }
        *reinterpret_cast<uint4*>(zbuf + p * zslot + zp * zplane + (size_t)(c * q.zrows + j) * 16) =
            make_uint4(wd[0], wd[1], wd[2], wd[3]);
      }
      // TSS = sum (T*m)^2 (m = 1 unmasked) of each rebuilt member, exact;
      // per-warp partials in shared memory
      for (uint32_t p = 0; p < nset; ++p) {
        if (!((zbits >> p) & 1u)) continue;
        const uint8_t* tp = P[pi + p].tpl;
        const uint8_t* mk = P[pi + p].mask;
        unsigned long long t2 = 0;
        for (uint32_t k = threadIdx.x; k < q.w * q.h; k += kThreads) {
          uint32_t t = __ldg(tp + k);
          if constexpr (MASKED) t *= __ldg(mk + k);
          t2 += (unsigned long long)t * t;
        }
        for (int o = 16; o > 0; o >>= 1) t2 += __shfl_down_sync(0xffffffffu, t2, o);
        if (lane == 0) s_part[p * kWarps + warp] = t2;
      }
    }
    if (zbits) {
      // the MMA band of every image row r of a tile: image row r feeds output
      // rows n in [r-h+1, r], rounded out to 16 (rows past the map are computed,
      // not stored): {first accumulator column n0, instruction descriptor with
      // N = n1 - n0, first Z row of the band}
      for (uint32_t r = threadIdx.x; r < q.rows_max; r += kThreads) {
        const uint32_t n0 = (r + 1 > q.h ? r + 1 - q.h : 0u) & ~15u;
        const uint32_t n1 = min(L.NT, (r & ~15u) + 16u);
        const uint32_t idesc = (idesc_u8u8_s32(kM, 16) & ~(0x3Fu << 17)) | (((n1 - n0) >> 3) << 17);
        reinterpret_cast<uint4*>(smem + kBandTable)[r] = make_uint4(n0, idesc, n0 + q.h + 15u - r, 0u);
      }
      fence_proxy_async_smem();
    }
    cp_async_wait_all();
    __syncthreads();
    if (*s_err) break;
    next = *s_next;
    if (zbits && threadIdx.x == 0) {
      // every thread has read the slots' keys above, before the barrier
      for (uint32_t p = 0; p < nset; ++p) {
        if (!((zbits >> p) & 1u)) continue;
        unsigned long long t = 0;
        for (int k = 0; k < kWarps; ++k) t += s_part[p * kWarps + k];
        s_tss[p] = (uint32_t)t;  // < 2^31: at most 33025 template pixels
        const UmmaProblem& mp = P[pi + p];
        s_zkey[p] = ZKey{mp.tpl, mp.mask, mp.w, mp.h, mp.kmma, 0u};
      }
    }
    // masked CrossCorrelation scores X alone: its members skip the Y
    // correlations, and a set of such members skips the I^2 planes
    uint32_t ymask = 0;  // members that need Y
    for (uint32_t p = 0; p < nset; ++p)
      if (!MASKED || P[pi + p].method != kCcorr) ymask |= 1u << p;
    const bool need_y = ymask != 0;
    if (MASKED && need_y) {
      // the two u8 parts of I^2 (I^2 mod 255, floor(I^2 / 255)) next to the
      // staged image
      const uint32_t words = nrows * L.imgp / 4;
      const uint32_t* i4 = reinterpret_cast<const uint32_t*>(img_buf);
      uint32_t* rem4 = reinterpret_cast<uint32_t*>(img_buf + L.plane_bytes);
      uint32_t* quo4 = reinterpret_cast<uint32_t*>(img_buf + 2 * L.plane_bytes);
      for (uint32_t idx = threadIdx.x; idx < words; idx += kThreads) {
        const uint32_t v = i4[idx];
        uint32_t rem = 0, quo = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t b = (v >> (8 * k)) & 0xFFu;
          const uint32_t sq = b * b;
          const uint32_t qd = sq / 255u;  // 0..255
          rem |= (sq - 255u * qd) << (8 * k);
          quo |= qd << (8 * k);
        }
        rem4[idx] = rem;
        quo4[idx] = quo;
      }
      __syncthreads();
    }
    // the next tile's rows stream into the other buffer during this tile
    if (L.nbuf == 2 && next < L.tiles) {
      const uint32_t pn = find_problem(L, P, pi, next);
      issue_tile_load(L, P[pn], s_img + (buf ^ 1u) * NPL * L.plane_bytes, next - P[pn].tile_begin);
    }
    const uint32_t nst = (nrows + L.rps - 1) / L.rps;
    const unsigned long long deadline = global_ns() + L.wait_ns;

    if (!mma_warp) {
      // builder warp: lane quadrant q4 of tensor memory, sub-group sub (kSubs per quadrant)
      const uint32_t q4 = warp & 3, sub = warp >> 2;
      const uint32_t m = q4 * 32 + lane;
      const uint32_t lane_base = q4 * 32;
      // accumulator columns this warp zeroes and finishes: the tile's 16-column
      // chunks shared out over the quadrant's kSubs warps (unevenly when NT / 16
      // is not a multiple of kSubs)
      const uint32_t chunks = L.NT / 16;
      const uint32_t c_begin = 16 * (sub * chunks / kSubs);
      const uint32_t ncols = 16 * ((sub + 1) * chunks / kSubs) - c_begin;
      {
        const uint32_t zero16[16] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        for (uint32_t p = 0; p <= nset; ++p) {
          if (p == nset && !MASKED) break;
          const uint32_t base = p < nset ? p * L.NT : ycol;  // members' X, then the set's Y
          for (uint32_t col = c_begin; col < c_begin + ncols; col += 16)
            tmem_st16(tmem_addr(tmem, lane_base, base + col), zero16);
        }
      }
      for (uint32_t st = 0; st < nst; ++st, ++g) {
        const uint32_t s = g % kStages;
        const bool got = g < kStages || mbar_wait_sleep(&empty[s], ((g / kStages) + 1) & 1u, deadline);
        if (!__all_sync(0xffffffffu, got)) {  // warp-uniform: the warp arrives as one below
          tmem_wait_st();  // the tile's zeroing stores land before tensor memory can be freed
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t r0 = st * L.rps, r_end = min(nrows, r0 + L.rps);
        // rows r == sub (mod kSubs) of this stage; the quadrant picks the
        // compile-time word offset of the lanes' windows (warp-uniform)
        const StageRows sr{img_buf, r0 + ((sub + kSubs - (r0 % kSubs)) % kSubs), r_end, r0,
                           a_col0 + s * L.rps * a_row_cols, a_row_cols, L.imgp, L.plane_bytes,
                           (uint32_t)lane, m, q.w, tmem, sub, s_rs, need_y};
        switch (q4) {
          case 0: build_stage_rows<KS, MASKED, 0>(sr); break;
          case 1: build_stage_rows<KS, MASKED, 1>(sr); break;
          case 2: build_stage_rows<KS, MASKED, 2>(sr); break;
          default: build_stage_rows<KS, MASKED, 3>(sr); break;
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&full[s]);
      }
      if (ok && !mbar_wait_sleep(dfull, tcount & 1u, deadline)) ok = false;
      // all builder threads reach this (every wait above is bounded): the row
      // sums written by the other builder warps are visible after it
      asm volatile("bar.sync 1, %0;" ::"n"(kBuilders) : "memory");
      if (ok) {
        tc_fence_after();
        const uint32_t x = x0 + lane_column(m);
        uint32_t Y = 0;  // window sums stay below 2^31 on this path
        if constexpr (!MASKED) {
          uint32_t y4[4] = {0u, 0u, 0u, 0u};
          uint32_t r = c_begin;
          for (; r + 4 <= c_begin + q.h; r += 4)
#pragma unroll
            for (int k = 0; k < 4; ++k) y4[k] += (r + k < nrows) ? s_rs[(r + k) * kM + m] : 0u;
          for (; r < c_begin + q.h; ++r) y4[0] += r < nrows ? s_rs[r * kM + m] : 0u;
          Y = y4[0] + y4[1] + y4[2] + y4[3];
        }
        // each member's scores from its own accumulators (Y is the members'
        // common window sum of I^2, unmasked)
        for (uint32_t p = 0; p < nset; ++p) {
          const UmmaProblem qp = P[pi + p];
          const UmmaEpi e{&qp, tmem, p * L.NT, ycol, lane_base, c_begin, ncols, L.NT, nrows, m, x, y0, s_tss[p],
                          (uint32_t)lane, s_rs, Y};
          umma_epilogue_dispatch<MASKED>(e, qp.method, qp.precision == IPB_PRECISION_EXACT_FP64, qp.ext != nullptr);
        }
      }
      if (!ok) {
        *s_err = 1;
        atomicMax(L.err, L.tag);
      }
    } else {
      // MMA warp: the whole warp runs the issue loop with warp-uniform values;
      // one elected lane issues each tcgen05.mma and commit
      const uint64_t desc0 = smem_desc_noswizzle(smem_u32(zbuf), q.zrows * 16, 128);
      const uint32_t dlo = (uint32_t)desc0, dhi = (uint32_t)(desc0 >> 32);
      const uint32_t zoff1 = zplane >> 4;
      const uint32_t zslot16 = zslot >> 4;   // one member's template side, in 16-byte units
      const uint32_t kstride = 2u * q.zrows;  // one 32-byte K step of Z, in 16-byte units
      const uint32_t ksteps = q.kmma / 32;
      const uint4* band = reinterpret_cast<const uint4*>(smem + kBandTable);
      const bool leader = elect_one();
      // test hook: a wait on the drain barrier, which nothing arrives at before the end
      if (L.stall && !__all_sync(0xffffffffu, mbar_wait(drain, 0, deadline))) ok = false;
      for (uint32_t st = 0; ok && st < nst; ++st, ++g) {
        const uint32_t s = g % kStages;
        const bool got = mbar_wait(&full[s], (g / kStages) & 1u, deadline);
        if (!__all_sync(0xffffffffu, got)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t r0 = st * L.rps, cnt = min(nrows, r0 + L.rps) - r0;
        const uint32_t a_stage = tmem + a_col0 + s * L.rps * a_row_cols;
        if (leader) {
          const StageIssue si{band, r0, cnt, a_stage, a_row_cols, dlo, dhi, zslot16, zoff1, kstride, ksteps,
                              tmem, L.NT, ycol, ymask};
          if constexpr (SETS) {
            switch (nset) {
              case 1: issue_stage<1, KS, MASKED>(si); break;
              case 2: issue_stage<2, KS, MASKED>(si); break;
              case 3: issue_stage<3, KS, MASKED>(si); break;
              default: issue_stage<4, KS, MASKED>(si); break;
            }
          } else {
            issue_stage<1, KS, MASKED>(si);
          }
          mma_commit(&empty[s]);
        }
        __syncwarp();
      }
      if (ok && leader) mma_commit(dfull);
      if (!ok && lane == 0) {
        *s_err = 1;
        atomicMax(L.err, L.tag);
      }
      __syncwarp();
    }
  }

  // drain outstanding copies and MMAs, then free tensor memory
  cp_async_wait_all();
  __syncthreads();
  if (L.sched && threadIdx.x == 0) {
    // every CTA has made its last claim before it counts itself out, so the
    // last one out re-arms the counter for the next launch that uses it
    __threadfence();
    if (atomicAdd(L.sched + 1, 1u) == gridDim.x - 1) {
      atomicExch(L.sched, 0u);
      atomicExch(L.sched + 1, 0u);
    }
  }
  if (mma_warp) {
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kWaitNs) && lane == 0) atomicMax(L.err, L.tag);
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

template <int KS, bool MASKED, bool SETS>
cudaError_t launch_ks(const UmmaLaunch& L, uint32_t smem, uint32_t grid, cudaStream_t s) {
  static PerDeviceOnce attr;  // per instantiation and device
  cudaError_t e = attr.run([] {
    return cudaFuncSetAttribute(umma_match_kernel<KS, MASKED, SETS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                227 * 1024);
  });
  if (e != cudaSuccess) return e;
  umma_match_kernel<KS, MASKED, SETS><<<grid, kThreads, smem, s>>>(L);
  return cudaGetLastError();
}

template <int KS, bool MASKED>
cudaError_t launch_ks2(const UmmaLaunch& L, uint32_t smem, uint32_t grid, cudaStream_t s) {
  return L.set_max > 1 ? launch_ks<KS, MASKED, true>(L, smem, grid, s) : launch_ks<KS, MASKED, false>(L, smem, grid, s);
}

template <int KS, bool MASKED>
cudaError_t set_smem_attr() {
  cudaError_t e = cudaFuncSetAttribute(umma_match_kernel<KS, MASKED, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(umma_match_kernel<KS, MASKED, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              227 * 1024);
}

int sm_count() { return device_sm_count(); }

uint32_t ks_of(uint32_t w) {
  const uint32_t kmma = (w + 31) & ~31u;
  uint32_t ks = 8;
  while (ks * 4 < kmma) ks *= 2;
  return ks;
}

// Kernel-wide tile and shared-memory plan for a group sharing (ks, masked):
// sized for the group's tallest template.
// nt_only: a tile height the plan must use (0: the tallest that fits).
// Tile heights, tallest first, for sets of up to `set` problems: a tile of
// NT output rows reads NT + h - 1 image rows, so taller tiles repeat fewer
// rows, while each member's accumulator (NT columns, plus the set's common Y
// with a mask) leaves less tensor memory for the A stages. Binary-mask tiles of 96 rows (`tall`:
// launches of many tiles, where throughput counts) only where a stage still
// holds 3 image rows; a launch of one map or one row band ends after about
// one tile's time, which the 64-row tile keeps shorter. Sets trade tile
// height for members: the A rows of a tile serve every member.
uint32_t tile_heights(bool masked, bool tall, uint32_t set, uint32_t out[2]) {
  if (set <= 1) {
    out[0] = masked ? (tall ? 96u : 64u) : 128u;
    out[1] = 64u;
  } else if (set == 2) {
    out[0] = masked ? 64u : 128u;
    out[1] = masked ? 32u : 64u;
  } else {
    out[0] = 64u;
    out[1] = 32u;
  }
  return 2;
}

bool make_plan(uint32_t ks, bool masked, uint32_t hmax, bool tall, UmmaPlan& pl, uint32_t nt_only = 0,
               uint32_t set = 1) {
  if (set < 1 || set > kMaxSet) return false;
  const uint32_t npl = masked ? 3 : 1, nz = masked ? 3 : 1;
  pl.ks = ks;
  pl.masked = masked;
  pl.set_max = set;
  pl.imgp = kM + 4 * ks + 16;
  const uint32_t kmma = 4 * ks;  // largest K of the group
  const uint32_t zplane = (kmma / 16) * (hmax + 32) * 16;
  uint32_t nts[2];
  tile_heights(masked, tall, set, nts);
  for (uint32_t nt : nts) {
    if (nt_only && nt != nt_only) continue;
    const uint32_t acc = (set + (masked ? 1u : 0u)) * nt;  // members' X, the set's Y
    if (acc >= kTmemCols) continue;
    const uint32_t tm_left = kTmemCols - acc;
    const uint32_t rps = tm_left / (kStages * npl * ks);
    if (rps < 1) continue;
    if (masked && nt > 64 && rps < 3) continue;
    const uint32_t rows = nt + hmax - 1;
    const uint32_t plane = (uint32_t)align_up((size_t)rows * pl.imgp, 128);
    for (uint32_t nbuf : {2u, 1u}) {
      const uint32_t z_off = kSmemHeader;
      const uint32_t img_off = z_off + (uint32_t)align_up((size_t)set * nz * zplane, 128);
      const uint32_t rs_off = img_off + nbuf * npl * plane;
      const uint32_t end = rs_off + (masked ? 0u : rows * kM * 4);
      if (end <= 227u * 1024u) {
        pl.NT = nt;
        pl.rps = rps > kMaxRps ? kMaxRps : rps;
        pl.plane_bytes = plane;
        pl.nbuf = nbuf;
        pl.z_off = z_off;
        pl.img_off = img_off;
        pl.rs_off = rs_off;
        pl.smem = end < kMinSmem ? kMinSmem : end;
        return true;
      }
    }
  }
  return false;
}

// Template shapes the tensor path takes: at least 8 columns (templates of
// 8..15 columns fill half of the first 32-byte K step, zeros the rest) and
// one 8-row band; rows within the band table; s32 sums exact (33025 pixels).
bool umma_shape_ok(uint32_t w, uint32_t h, bool masked) {
  return w >= 8 && h >= 8 && h <= 128 && w <= (masked ? 128u : 256u) && (size_t)w * h <= 33025;
}

}  // namespace

bool umma_supported(const MatchArgs& a) {
  if (a.precision == IPB_PRECISION_REFERENCE_F32) return false;
  if (a.mask && !a.mask_binary) return false;  // general u8 masks: CUDA-core byte planes
  if (!umma_shape_ok(a.w, a.h, a.mask != nullptr)) return false;
  UmmaPlan pl;
  return make_plan(ks_of(a.w), a.mask != nullptr, a.h, /*tall=*/false, pl);
}

uint32_t umma_group_key(const MatchArgs& a) { return ks_of(a.w) * 2 + (a.mask ? 1 : 0); }
uint32_t umma_row_width(uint32_t w) { return ks_of(w); }

cudaError_t umma_prepare_kernels() {
  cudaError_t e;
  if ((e = set_smem_attr<8, false>()) != cudaSuccess || (e = set_smem_attr<16, false>()) != cudaSuccess ||
      (e = set_smem_attr<32, false>()) != cudaSuccess || (e = set_smem_attr<64, false>()) != cudaSuccess ||
      (e = set_smem_attr<8, true>()) != cudaSuccess || (e = set_smem_attr<16, true>()) != cudaSuccess ||
      (e = set_smem_attr<32, true>()) != cudaSuccess)
    return e;
  return cudaSuccess;
}

bool umma_plan_for(uint32_t ks, bool masked, uint32_t hmax, UmmaPlan& pl, uint32_t nt, uint32_t set) {
  if (ks < 8 || ks > (masked ? 32u : 64u) || (ks & (ks - 1))) return false;
  return make_plan(ks, masked, hmax, /*tall=*/true, pl, nt, set);
}

uint32_t umma_tile_heights(bool masked, uint32_t set, uint32_t out[2]) {
  return tile_heights(masked, /*tall=*/true, set, out);
}

namespace {
// the class a problem's set is drawn from: one image, one template size, one mask kind
// (binary-mask sets also share the mask buffer: their Y is common)
bool same_class(const UmmaProblem& a, const UmmaProblem& b) {
  return a.img == b.img && a.W == b.W && a.H == b.H && a.w == b.w && a.h == b.h && a.mask == b.mask;
}
bool class_less(const UmmaProblem& a, const UmmaProblem& b) {
  return std::tie(a.img, a.W, a.H, a.w, a.h, a.mask) < std::tie(b.img, b.W, b.H, b.w, b.h, b.mask);
}
}  // namespace

uint32_t umma_largest_set(const std::vector<UmmaProblem>& probs) {
  std::vector<UmmaProblem> v(probs);
  std::stable_sort(v.begin(), v.end(), class_less);
  uint32_t best = v.empty() ? 0u : 1u;
  for (size_t i = 0, j; i < v.size(); i = j) {
    for (j = i + 1; j < v.size() && same_class(v[i], v[j]); ++j) {
    }
    best = std::max(best, (uint32_t)(j - i));
  }
  return std::min(best, kMaxSet);
}

uint32_t umma_make_sets(std::vector<UmmaProblem>& probs, const UmmaPlan& pl) {
  std::stable_sort(probs.begin(), probs.end(), class_less);
  uint32_t tiles = 0;
  for (size_t i = 0, j; i < probs.size(); i = j) {
    for (j = i + 1; j < probs.size() && same_class(probs[i], probs[j]); ++j) {
    }
    // a class of cnt problems in nsets sets whose sizes differ by at most one
    const uint32_t cnt = (uint32_t)(j - i), cap = std::max(pl.set_max, 1u);
    const uint32_t nsets = (cnt + cap - 1) / cap;
    size_t k = i;
    for (uint32_t t = 0; t < nsets; ++t) {
      const uint32_t sz = cnt / nsets + (t < cnt % nsets ? 1u : 0u);
      for (uint32_t u = 0; u < sz; ++u) {
        probs[k + u].set_n = u == 0 ? sz : 0u;
        probs[k + u].tile_begin = tiles;
      }
      tiles += umma_problem_tiles(probs[k], pl);
      k += sz;
    }
  }
  return tiles;
}

UmmaProblem umma_problem(const MatchArgs& a, const UmmaPlan& pl, uint32_t tile_begin,
                         unsigned long long* ext_keys) {
  UmmaProblem q{};
  q.img = a.img;
  q.tpl = a.tpl;
  q.mask = a.mask;
  q.out = a.out;
  q.ext = ext_keys;
  q.W = a.W;
  q.H = a.H;
  q.w = a.w;
  q.h = a.h;
  q.Wo = a.W - a.w + 1;
  q.Ho = a.H - a.h + 1;
  q.tiles_x = (q.Wo + kM - 1) / kM;
  q.tile_begin = tile_begin;
  q.kmma = (a.w + 31) & ~31u;
  q.zrows = a.h + 32;
  q.rows_max = pl.NT + a.h - 1;
  const uintptr_t ia = reinterpret_cast<uintptr_t>(a.img);
  q.load_mode = ((ia & 15u) == 0 && (a.W & 15u) == 0) ? 2 : (((ia & 3u) == 0 && (a.W & 3u) == 0) ? 1 : 0);
  q.method = a.method;
  q.precision = a.precision;
  q.set_n = 1;
  return q;
}

uint32_t umma_problem_tiles(const UmmaProblem& q, const UmmaPlan& pl) {
  return q.tiles_x * ((q.Ho + pl.NT - 1) / pl.NT);
}

cudaError_t launch_umma_batch(const UmmaPlan& pl, UmmaLaunch& L, cudaStream_t stream, KernelTimer* timer) {
  L.NT = pl.NT;
  L.rps = pl.rps;
  L.imgp = pl.imgp;
  L.plane_bytes = pl.plane_bytes;
  L.nbuf = pl.nbuf;
  L.z_off = pl.z_off;
  L.img_off = pl.img_off;
  L.rs_off = pl.rs_off;
  L.set_max = pl.set_max;
  if (L.tiles == 0) return cudaSuccess;
  const uint32_t grid = L.tiles < (uint32_t)sm_count() ? L.tiles : (uint32_t)sm_count();
  cudaError_t e;
  timer_begin(timer, kKernelUmma, stream);
  if (pl.masked) {
    switch (pl.ks) {
      case 8: e = launch_ks2<8, true>(L, pl.smem, grid, stream); break;
      case 16: e = launch_ks2<16, true>(L, pl.smem, grid, stream); break;
      default: e = launch_ks2<32, true>(L, pl.smem, grid, stream); break;
    }
  } else {
    switch (pl.ks) {
      case 8: e = launch_ks2<8, false>(L, pl.smem, grid, stream); break;
      case 16: e = launch_ks2<16, false>(L, pl.smem, grid, stream); break;
      case 32: e = launch_ks2<32, false>(L, pl.smem, grid, stream); break;
      default: e = launch_ks2<64, false>(L, pl.smem, grid, stream); break;
    }
  }
  count_launch(kKernelUmma);
  timer_end(timer, stream);
  return e;
}

cudaError_t launch_umma_extremes(const uint8_t* img, uint32_t W, uint32_t H, const uint8_t* const* tpls,
                                 uint32_t n, uint32_t w, uint32_t h, int method, int precision,
                                 unsigned long long* keys, unsigned int* err_word, unsigned int tag,
                                 cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (n > kInlineProblems || !umma_shape_ok(w, h, false)) return cudaErrorNotSupported;
  // the templates share the image: sets of up to kMaxSet share its A rows
  const uint32_t nsets = (n + kMaxSet - 1) / kMaxSet, set = (n + nsets - 1) / nsets;
  UmmaPlan pl;
  if (!make_plan(ks_of(w), false, h, /*tall=*/true, pl, 0, set) && !make_plan(ks_of(w), false, h, true, pl, 0, 1))
    return cudaErrorNotSupported;
  cudaError_t e = umma_prepare_kernels();
  if (e != cudaSuccess) return e;
  std::vector<UmmaProblem> probs;
  for (uint32_t i = 0; i < n; ++i) {
    const MatchArgs a{img, W, H, tpls[i], w, h, nullptr, false, method, precision, nullptr, stream};
    probs.push_back(umma_problem(a, pl, 0, keys + 2 * i));
  }
  const uint32_t tiles = umma_make_sets(probs, pl);
  UmmaLaunch L{};
  for (uint32_t i = 0; i < n; ++i) L.inl[i] = probs[i];
  L.nprobs = n;
  L.tiles = tiles;
  L.err = err_word;
  L.tag = tag;
  L.wait_ns = pipeline_wait_ns();
  L.stall = pipeline_stall() ? 1u : 0u;
  return launch_umma_batch(pl, L, stream, nullptr);
}

cudaError_t launch_umma(const MatchArgs& a, unsigned int* err_word, unsigned int tag) {
  UmmaPlan pl;
  if (!make_plan(ks_of(a.w), a.mask != nullptr, a.h, /*tall=*/false, pl)) return cudaErrorNotSupported;
  UmmaLaunch L{};
  L.inl[0] = umma_problem(a, pl, 0, nullptr);
  L.nprobs = 1;
  L.tiles = umma_problem_tiles(L.inl[0], pl);
  L.err = err_word;
  L.tag = tag;
  L.wait_ns = pipeline_wait_ns();
  L.stall = pipeline_stall() ? 1u : 0u;
  return launch_umma_batch(pl, L, a.stream, a.timer);
}

// ---- fused find_extremes bookkeeping ---------------------------------------
__global__ void extremes_keys_init_kernel(unsigned long long* keys, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    keys[2 * i] = ~0ull;
    keys[2 * i + 1] = 0ull;
  }
}

// keys -> ipb_extremes_f32 (the order key inverts exactly; indices -> (x, y))
// Writes the records and re-arms the keys ({~0, 0}) for the next launch
// of the same plan, so a replayed batch needs no separate initialisation.
__global__ void extremes_keys_finish_kernel(unsigned long long* keys, const uint32_t* widths,
                                            ipb_extremes_f32* const* outs, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long kmin = keys[2 * i], kmax = keys[2 * i + 1];
  keys[2 * i] = ~0ull;
  keys[2 * i + 1] = 0ull;
  if (!outs[i]) return;
  auto value = [](uint32_t ok) {
    const uint32_t b = (ok & 0x80000000u) ? (ok & 0x7FFFFFFFu) : ~ok;
    return __uint_as_float(b);
  };
  const uint32_t imin = (uint32_t)kmin, imax = 0xFFFFFFFFu - (uint32_t)kmax;
  ipb_extremes_f32 r;
  r.max_value = value((uint32_t)(kmax >> 32));
  r.min_value = value((uint32_t)(kmin >> 32));
  r.max_value_location_x = imax % widths[i];
  r.max_value_location_y = imax / widths[i];
  r.min_value_location_x = imin % widths[i];
  r.min_value_location_y = imin / widths[i];
  *outs[i] = r;
}

cudaError_t launch_extremes_keys_init(unsigned long long* keys, uint32_t n, cudaStream_t s) {
  if (!n) return cudaSuccess;
  extremes_keys_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(keys, n);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

cudaError_t launch_extremes_keys_finish(unsigned long long* keys, const uint32_t* widths,
                                        ipb_extremes_f32* const* outs, uint32_t n, cudaStream_t s) {
  if (!n) return cudaSuccess;
  extremes_keys_finish_kernel<<<(n + 255) / 256, 256, 0, s>>>(keys, widths, outs, n);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

}  // namespace ipb

#define IPB_API extern "C" __attribute__((visibility("default")))

IPB_API ipb_status ipb_tensor_set_plan_for(uint32_t w, uint32_t h, int masked, uint32_t problems_per_set,
                                           ipb_tensor_plan* out) {
  using namespace ipb;
  if (!out) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null argument");
  if (!umma_shape_ok(w, h, masked != 0))
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "template shape not taken by the tensor path");
  if (problems_per_set < 1 || problems_per_set > kMaxSet)
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "problems per set outside 1..4");
  UmmaPlan pl;
  if (!make_plan(ks_of(w), masked != 0, h, /*tall=*/true, pl, 0, problems_per_set))
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "no tensor-core plan fits this template");
  const uint32_t planes = masked ? 3u : 1u, accumulators = masked ? 2u : 1u;
  out->tile_rows = pl.NT;
  out->image_rows = pl.NT + h - 1;
  out->rows_per_stage = pl.rps;
  out->stages = kStages;
  out->image_buffers = pl.nbuf;
  out->tmem_columns = (problems_per_set + accumulators - 1) * pl.NT + kStages * planes * pl.ks * pl.rps;
  out->smem_bytes = pl.smem;
  return IPB_OK;
}

IPB_API ipb_status ipb_tensor_plan_for(uint32_t w, uint32_t h, int masked, int batch, ipb_tensor_plan* out) {
  using namespace ipb;
  if (!out) return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null argument");
  if (!umma_shape_ok(w, h, masked != 0))
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "template shape not taken by the tensor path");
  UmmaPlan pl;
  if (!make_plan(ks_of(w), masked != 0, h, batch != 0, pl))
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "no tensor-core plan fits this template");
  const uint32_t planes = masked ? 3u : 1u, accumulators = masked ? 2u : 1u;
  out->tile_rows = pl.NT;
  out->image_rows = pl.NT + h - 1;
  out->rows_per_stage = pl.rps;
  out->stages = kStages;
  out->image_buffers = pl.nbuf;
  out->tmem_columns = accumulators * pl.NT + kStages * planes * pl.ks * pl.rps;
  out->smem_bytes = pl.smem;
  return IPB_OK;
}
