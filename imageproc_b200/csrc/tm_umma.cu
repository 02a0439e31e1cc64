// tm_umma.cu -- exact template matching on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, unsigned u8 x u8 -> s32, accumulators in tensor memory).
//
// Replaces the scalar walk of methods::*::score_at (src/template_matching.rs:
// 219-376) for unmasked and binary-masked matches with templates up to
// 256 x 128 pixels (128 x 128 masked).
//
// Formulation. A CTA owns a tile of 128 output columns (x0 + m, m = tensor-
// memory lane) by NT output rows (y0 + n, n = tensor-memory column). For each
// image row r of the tile (r = 0 .. NT + h - 2, image row y0 + r) and each
// correlation c:
//   A_r[m][k] = P_c[y0 + r][x0 + m + k]          (a Hankel row per lane)
//   B_r[n][k] = Q_c[r - n][k]                     (0 <= r - n < h, else 0)
//   D_c[m][n] += sum_k A_r[m][k] * B_r[n][k]
// so that after all rows D_c[m][n] = sum_{dy,dx} P_c[y0+n+dy][x0+m+dx] Q_c[dy][dx].
//   unmasked:     c = 0: P = I, Q = T                          -> X
//   binary mask:  c = 0: P = I, Q = T*m                        -> X
//                 c = 1: P = low byte of I^2,  Q = m           \ Y = D_1 + 256 D_2
//                 c = 2: P = high byte of I^2, Q = m           /
// B_r is a window of one buffer Z_c (Q_c with its rows reversed and 16 zero
// rows on each side) stored in the canonical no-swizzle K-major layout, whose
// rows are 16 bytes apart: moving from r to r+1 moves B's start address by
// -16 bytes. Only the 16-aligned band of n where B_r is non-zero is issued.
//
// A_r goes straight into tensor memory: eight builder warps form each lane's
// K bytes from the staged image rows with byte_perm and store them with
// tcgen05.st (the MMA reads A from tensor memory and only B from shared
// memory). Unmasked, the same words give the lane's row sum of squares with
// dp4a, from which the epilogue slides the window sum Y = sum I^2 over h rows,
// so no integral image is needed. The kernel also builds Z and the template
// constant TSS from the raw template (and mask) itself: a call is one launch.
//
// Pipeline: image tiles are double-buffered in shared memory and loaded with
// cp.async while the previous tile is computed. Builders fill 3 stages of RPS
// A rows; one thread issues the MMAs of a stage from a per-tile table once the
// stage is full and commits it back to the builders; after the tile's last
// stage it commits the accumulators to the epilogue (the builder warps), which
// reads them with tcgen05.ld and writes the scores. Every wait is bounded
// (2 s); a wait that runs out records the launch's tag in the error word and
// the CTA leaves its loop, drains its MMAs and frees its tensor memory.
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
constexpr int kStages = 3;
constexpr uint32_t kMaxRps = 16;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr uint32_t kSmemHeader = 1024;
constexpr uint32_t kMinSmem = 120 * 1024;  // keeps residency at one CTA per SM

struct UmmaParams {
  const uint8_t* img;
  uint32_t W, H;
  const uint8_t* tpl;   // raw template, w x h
  const uint8_t* mask;  // raw binary mask or null
  uint32_t w, h;
  uint32_t kmma;      // K of the MMAs: w rounded up to 32
  uint32_t NT;        // output rows per tile
  uint32_t rps;       // image rows per pipeline stage
  uint32_t imgp;      // staged image row pitch (bytes)
  uint32_t rows_max;  // NT + h - 1
  uint32_t zrows;     // rows of a reversed-template buffer: h + 32
  uint32_t zplane;    // bytes of one reversed-template buffer
  uint32_t tab_off, z_off, img_off, rs_off;  // shared-memory carve
  uint32_t plane_bytes;  // one staged image plane: rows_max * imgp
  uint32_t nbuf;         // staged image buffers (1 or 2)
  uint32_t Wo, Ho, tiles_x, tiles;
  int method, precision, load_mode;  // load_mode: 2 = cp.async 16 B, 1 = 4 B, 0 = plain loads
  float* out;
  unsigned int* err;
  unsigned int tag;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Stage image rows [y0, y0 + nrows) x columns [x0, x0 + imgp) of plane 0,
// zero past the right edge. Asynchronous unless load_mode == 0.
__device__ void issue_tile_load(const UmmaParams& p, uint8_t* dst_plane, uint32_t tile) {
  const uint32_t x0 = (tile % p.tiles_x) * kM;
  const uint32_t y0 = (tile / p.tiles_x) * p.NT;
  const uint32_t nrows = min(p.rows_max, p.H - y0);
  const uint8_t* src = p.img + (size_t)y0 * p.W;
  if (p.load_mode == 2) {
    const uint32_t chunks = p.imgp / 16;
    for (uint32_t idx = threadIdx.x; idx < nrows * chunks; idx += kThreads) {
      const uint32_t r = idx / chunks, c = (idx % chunks) * 16, gx = x0 + c;
      const uint32_t avail = gx < p.W ? min(16u, p.W - gx) : 0u;
      const uint8_t* g = src + (size_t)r * p.W + (avail ? gx : 0u);
      cp_async16(smem_u32(dst_plane + r * p.imgp + c), g, avail);
    }
  } else if (p.load_mode == 1) {
    const uint32_t words = p.imgp / 4;
    for (uint32_t idx = threadIdx.x; idx < nrows * words; idx += kThreads) {
      const uint32_t r = idx / words, c = (idx % words) * 4, gx = x0 + c;
      const uint32_t avail = gx < p.W ? min(4u, p.W - gx) : 0u;
      const uint8_t* g = src + (size_t)r * p.W + (avail ? gx : 0u);
      cp_async4(smem_u32(dst_plane + r * p.imgp + c), g, avail);
    }
  } else {
    const uint32_t words = p.imgp / 4;
    for (uint32_t idx = threadIdx.x; idx < nrows * words; idx += kThreads) {
      const uint32_t r = idx / words, c = (idx % words) * 4, gx = x0 + c;
      const uint8_t* row = src + (size_t)r * p.W;
      uint32_t v = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (gx + k < p.W) v |= (uint32_t)__ldg(row + gx + k) << (8 * k);
      *reinterpret_cast<uint32_t*>(dst_plane + r * p.imgp + c) = v;
    }
  }
  cp_async_commit();
}

// Builds one A row (one plane) for lane m into tensor memory; returns the
// lane's row sum of squares over the template width when kRowSums.
template <int KS, bool kRowSums>
__device__ __forceinline__ uint32_t build_row(const uint8_t* plane_row, uint32_t m, uint32_t w,
                                              uint32_t taddr) {
  const uint32_t* wp = reinterpret_cast<const uint32_t*>(plane_row) + (m >> 2);
  const uint32_t sel = 0x3210u + (m & 3u) * 0x1111u;
  uint32_t rs = 0;
  constexpr int CH = KS < 16 ? KS : 16;
  const uint32_t wq = w >> 2;
  const uint32_t tail = (w & 3u) ? ((1u << (8u * (w & 3u))) - 1u) : 0u;
#pragma unroll
  for (int c0 = 0; c0 < KS; c0 += CH) {
    uint32_t wv[CH + 1];
#pragma unroll
    for (int k = 0; k <= CH; ++k) wv[k] = wp[c0 + k];
    uint32_t a[CH];
#pragma unroll
    for (int k = 0; k < CH; ++k) a[k] = __byte_perm(wv[k], wv[k + 1], sel);
    if constexpr (kRowSums) {
      if (c0 + CH <= (int)wq) {
#pragma unroll
        for (int k = 0; k < CH; ++k) rs = __dp4a(a[k], a[k], rs);
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

template <int KS, bool MASKED>
__global__ void __launch_bounds__(kThreads, 1) umma_match_kernel(const UmmaParams p) {
  constexpr int NPL = MASKED ? 3 : 1;    // staged image planes: I (, low, high byte of I^2)
  constexpr int NCORR = MASKED ? 3 : 1;  // correlations / accumulators
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  uint64_t* dfull = empty + kStages;
  uint64_t* drain = dfull + 1;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + 128);
  volatile int* s_err = reinterpret_cast<volatile int*>(smem + 132);
  unsigned long long* s_tss = reinterpret_cast<unsigned long long*>(smem + 136);
  uint8_t* zbuf = smem + p.z_off;
  uint8_t* s_img = smem + p.img_off;
  uint32_t* s_rs = reinterpret_cast<uint32_t*>(smem + p.rs_off);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool mma_warp = warp == kBuilderWarps;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], kBuilders);
      mbar_init(&empty[s], 1);
    }
    mbar_init(dfull, 1);
    mbar_init(drain, 1);
    *s_err = 0;
    *s_tss = 0ull;
    mbar_init_fence();
  }
  if (mma_warp) {
    tmem_alloc(s_tmem, kTmemCols);
    tmem_relinquish();
  }
  // first tile's rows start streaming in while the template side is prepared
  if (blockIdx.x < p.tiles) issue_tile_load(p, s_img, blockIdx.x);
  __syncthreads();  // s_tss initialised
  // Z buffers, K-chunk-major: chunk c holds rows j = 0..zrows-1 of 16 bytes,
  // row j = template row h-1-(j-16) for 16 <= j < h+16, else zero.
  //   unmasked: Z_0 from T;  binary mask: Z_0 from T*m, Z_1 from m
  {
    constexpr int NZ = MASKED ? 2 : 1;
    const uint32_t nchunks = p.kmma / 16;
    for (uint32_t idx = threadIdx.x; idx < NZ * nchunks * p.zrows; idx += kThreads) {
      const uint32_t zp = idx / (nchunks * p.zrows);
      const uint32_t rem = idx % (nchunks * p.zrows);
      const uint32_t c = rem / p.zrows, j = rem % p.zrows;
      uint32_t wd[4] = {0u, 0u, 0u, 0u};
      if (j >= 16 && j < p.h + 16) {
        const size_t row = (size_t)(p.h - 1 - (j - 16)) * p.w;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const uint32_t dx = 16 * c + k;
          if (dx < p.w) {
            uint32_t v;
            if constexpr (MASKED) {
              const uint32_t mv = __ldg(p.mask + row + dx);
              v = zp == 0 ? (uint32_t)__ldg(p.tpl + row + dx) * mv : mv;
            } else {
              v = __ldg(p.tpl + row + dx);
            }
            wd[k >> 2] |= (v & 0xFFu) << (8 * (k & 3));
          }
        }
      }
      *reinterpret_cast<uint4*>(zbuf + zp * p.zplane + (size_t)(c * p.zrows + j) * 16) =
          make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
    // TSS = sum (T*m)^2 (m = 1 unmasked), exact in u64
    unsigned long long t2 = 0;
    for (uint32_t k = threadIdx.x; k < p.w * p.h; k += kThreads) {
      uint32_t t = __ldg(p.tpl + k);
      if constexpr (MASKED) t *= __ldg(p.mask + k);
      t2 += (unsigned long long)t * t;
    }
    for (int o = 16; o > 0; o >>= 1) t2 += __shfl_down_sync(0xffffffffu, t2, o);
    if (lane == 0 && t2) atomicAdd(s_tss, t2);
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t a_col0 = NCORR * p.NT;
  const uint32_t a_row_cols = NPL * KS;
  const uint32_t tss = (uint32_t)*s_tss;  // < 2^31: at most 33025 template pixels
  const uint64_t desc0 = smem_desc_noswizzle(smem_u32(zbuf), p.zrows * 16, 128);
  const uint32_t idesc0 = idesc_u8u8_s32(kM, 16) & ~(0x3Fu << 17);
  const uint32_t ksteps = p.kmma / 32;

  uint32_t g = 0;       // pipeline stage fills so far (same count in builders and the MMA thread)
  uint32_t tcount = 0;  // tiles finished by this CTA
  bool ok = true;

  for (uint32_t tile = blockIdx.x; tile < p.tiles; tile += gridDim.x, ++tcount) {
    __syncthreads();
    if (*s_err) break;
    const uint32_t buf = p.nbuf == 2 ? (tcount & 1u) : 0u;
    uint8_t* img_buf = s_img + buf * NPL * p.plane_bytes;
    if (p.nbuf == 1 && tcount > 0) issue_tile_load(p, img_buf, tile);
    const uint32_t x0 = (tile % p.tiles_x) * kM;
    const uint32_t y0 = (tile / p.tiles_x) * p.NT;
    const uint32_t nrows = min(p.rows_max, p.H - y0);
    cp_async_wait_all();
    __syncthreads();
    if (*s_err) break;
    if constexpr (MASKED) {
      // byte planes of I^2 next to the staged image
      const uint32_t words = nrows * p.imgp / 4;
      const uint32_t* i4 = reinterpret_cast<const uint32_t*>(img_buf);
      uint32_t* lo4 = reinterpret_cast<uint32_t*>(img_buf + p.plane_bytes);
      uint32_t* hi4 = reinterpret_cast<uint32_t*>(img_buf + 2 * p.plane_bytes);
      for (uint32_t idx = threadIdx.x; idx < words; idx += kThreads) {
        const uint32_t v = i4[idx];
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t b = (v >> (8 * k)) & 0xFFu;
          const uint32_t sq = b * b;
          lo |= (sq & 0xFFu) << (8 * k);
          hi |= (sq >> 8) << (8 * k);
        }
        lo4[idx] = lo;
        hi4[idx] = hi;
      }
      __syncthreads();
    }
    // the next tile's rows stream into the other buffer during this tile
    if (p.nbuf == 2 && tile + gridDim.x < p.tiles)
      issue_tile_load(p, s_img + (buf ^ 1u) * NPL * p.plane_bytes, tile + gridDim.x);
    const uint32_t nst = (nrows + p.rps - 1) / p.rps;
    const unsigned long long deadline = global_ns() + kWaitNs;

    if (!mma_warp) {
      // builder warp: lane quadrant q of tensor memory, sub-group sub (4 per quadrant)
      const uint32_t q = warp & 3, sub = warp >> 2;
      const uint32_t m = q * 32 + lane;
      const uint32_t lane_base = q * 32;
      const uint32_t ncols = p.NT / kSubs;  // accumulator columns this warp zeroes and finishes
      const uint32_t c_begin = sub * ncols;
      // zero this warp's share of the accumulators
      {
        const uint32_t zero16[16] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for (int c = 0; c < NCORR; ++c)
          for (uint32_t col = c_begin; col < c_begin + ncols; col += 16)
            tmem_st16(tmem_addr(tmem, lane_base, c * p.NT + col), zero16);
      }
      for (uint32_t st = 0; st < nst; ++st, ++g) {
        const uint32_t s = g % kStages;
        if (g >= kStages && !mbar_wait_sleep(&empty[s], ((g / kStages) + 1) & 1u, deadline)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t r0 = st * p.rps, r_end = min(nrows, r0 + p.rps);
        // rows r == sub (mod kSubs) of this stage
        for (uint32_t r = r0 + ((sub + kSubs - (r0 % kSubs)) % kSubs); r < r_end; r += kSubs) {
          const uint32_t tcol = a_col0 + (s * p.rps + (r - r0)) * a_row_cols;
          const uint8_t* row = img_buf + r * p.imgp;
          if constexpr (MASKED) {
#pragma unroll
            for (int pl = 0; pl < NPL; ++pl)
              build_row<KS, false>(row + pl * p.plane_bytes, m, p.w, tmem_addr(tmem, lane_base, tcol + pl * KS));
          } else {
            s_rs[r * kM + m] = build_row<KS, true>(row, m, p.w, tmem_addr(tmem, lane_base, tcol));
          }
        }
        tmem_wait_st();
        tc_fence_before();
        mbar_arrive(&full[s]);
      }
      if (ok && !mbar_wait_sleep(dfull, tcount & 1u, deadline)) ok = false;
      // all builder threads reach this (every wait above is bounded): the row
      // sums written by the other builder warps are visible after it
      asm volatile("bar.sync 1, %0;" ::"n"(kBuilders) : "memory");
      if (ok) {
        tc_fence_after();
        const uint32_t x = x0 + m;
        uint32_t Y = 0;  // window sums stay below 2^31 on this path
        if constexpr (!MASKED) {
          uint32_t y4[4] = {0u, 0u, 0u, 0u};
          uint32_t r = c_begin;
          for (; r + 4 <= c_begin + p.h; r += 4)
#pragma unroll
            for (int k = 0; k < 4; ++k) y4[k] += (r + k < nrows) ? s_rs[(r + k) * kM + m] : 0u;
          for (; r < c_begin + p.h; ++r) y4[0] += r < nrows ? s_rs[r * kM + m] : 0u;
          Y = y4[0] + y4[1] + y4[2] + y4[3];
        }
        for (uint32_t n0 = c_begin; n0 < c_begin + ncols; n0 += 16) {
          uint32_t vx[16];
          tmem_ld16(tmem_addr(tmem, lane_base, n0), vx);
          uint32_t vl[MASKED ? 16 : 1], vh[MASKED ? 16 : 1];
          uint32_t yv[16];
          if constexpr (MASKED) {
            tmem_ld16(tmem_addr(tmem, lane_base, p.NT + n0), vl);
            tmem_ld16(tmem_addr(tmem, lane_base, 2 * p.NT + n0), vh);
          } else {
            // window sums of the chunk: loads first, then the sliding chain
            uint32_t add[16], subv[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              const uint32_t ra = n0 + k + p.h, rb = n0 + k;
              add[k] = ra < nrows ? s_rs[ra * kM + m] : 0u;
              subv[k] = rb < nrows ? s_rs[rb * kM + m] : 0u;
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              yv[k] = Y;
              Y += add[k];
              Y -= subv[k];
            }
          }
          tmem_wait_ld();
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const uint32_t y = y0 + n0 + k;
            uint32_t Yk;
            if constexpr (MASKED) Yk = vl[k] + (vh[k] << 8);
            else Yk = yv[k];
            if (x < p.Wo && y < p.Ho)
              p.out[(size_t)y * p.Wo + x] = finish_score32(p.method, p.precision, vx[k], Yk, tss);
          }
        }
      }
      if (!ok) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    } else {
      // MMA warp: the whole warp runs the issue loop with warp-uniform values;
      // one elected lane issues each tcgen05.mma and commit
      const uint32_t dlo = (uint32_t)desc0, dhi = (uint32_t)(desc0 >> 32);
      const uint32_t zoff1 = p.zplane >> 4;
      const uint32_t kstride = 2u * p.zrows;  // one 32-byte K step of Z, in 16-byte units
      const bool leader = elect_one();
      for (uint32_t st = 0; st < nst; ++st, ++g) {
        const uint32_t s = g % kStages;
        const bool got = mbar_wait(&full[s], (g / kStages) & 1u, deadline);
        if (!__all_sync(0xffffffffu, got)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t r0 = st * p.rps, cnt = min(nrows, r0 + p.rps) - r0;
        const uint32_t a_stage = tmem + a_col0 + s * p.rps * a_row_cols;
        // image row r feeds output rows n in [r-h+1, r] of the tile: the band
        // [n0, n1) rounded out to 16 (rows past the map are computed, not stored)
#pragma unroll 4
        for (uint32_t i = 0; i < kMaxRps; ++i) {
          if (i >= cnt) break;
          const uint32_t r = r0 + i;
          const uint32_t n0 = (r + 1 > p.h ? r + 1 - p.h : 0u) & ~15u;
          const uint32_t n1 = min(p.NT, (r & ~15u) + 16u);
          const uint32_t idesc = idesc0 | (((n1 - n0) >> 3) << 17);
          const uint32_t zrow = dlo + n0 + p.h + 15u - r;  // first Z row of the band
          const uint32_t a = a_stage + i * a_row_cols;
          if (leader) {
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              const uint32_t zo = zrow + (c == 0 ? 0u : zoff1);
#pragma unroll
              for (uint32_t kk = 0; kk < (uint32_t)(KS / 8); ++kk) {
                if (kk < ksteps)
                  mma_i8_ts(tmem + c * p.NT + n0, a + (MASKED ? c * KS : 0) + kk * 8,
                            ((uint64_t)dhi << 32) | (zo + kk * kstride), idesc, 1u);
              }
            }
          }
        }
        if (leader) mma_commit(&empty[s]);
        __syncwarp();
      }
      if (ok && leader) mma_commit(dfull);
      if (!ok && lane == 0) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
      __syncwarp();
    }
  }

  // drain outstanding copies and MMAs, then free tensor memory
  cp_async_wait_all();
  __syncthreads();
  if (mma_warp) {
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kWaitNs) && lane == 0) atomicMax(p.err, p.tag);
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

struct Plan {
  uint32_t kmma, ks, NT, rps, imgp, rows_max, zrows, zplane, plane_bytes, nbuf;
  uint32_t tab_off, z_off, img_off, rs_off, smem;
};

bool make_plan(uint32_t w, uint32_t h, bool masked, Plan& pl) {
  if (w < 8 || w > (masked ? 128u : 256u) || h < 1 || h > 128) return false;
  const uint32_t npl = masked ? 3 : 1, ncorr = masked ? 3 : 1, nz = masked ? 2 : 1;
  pl.kmma = (w + 31) & ~31u;
  uint32_t ks = 8;
  while (ks * 4 < pl.kmma) ks *= 2;
  pl.ks = ks;
  pl.imgp = kM + 4 * ks + 16;
  pl.zrows = h + 32;
  pl.zplane = (pl.kmma / 16) * pl.zrows * 16;
  const uint32_t nts[2] = {masked ? 64u : 128u, 64u};
  for (uint32_t nt : nts) {
    const uint32_t tm_left = kTmemCols - ncorr * nt;
    const uint32_t rps = tm_left / (kStages * npl * ks);
    if (rps < 1) continue;
    const uint32_t rows = nt + h - 1;
    const uint32_t plane = (uint32_t)align_up((size_t)rows * pl.imgp, 128);
    for (uint32_t nbuf : {2u, 1u}) {
      const uint32_t tab_off = kSmemHeader;
      const uint32_t z_off = tab_off + (uint32_t)align_up(rows * 8, 128);
      const uint32_t img_off = z_off + (uint32_t)align_up((size_t)nz * pl.zplane, 128);
      const uint32_t rs_off = img_off + nbuf * npl * plane;
      const uint32_t end = rs_off + (masked ? 0u : rows * kM * 4);
      if (end <= 227u * 1024u) {
        pl.NT = nt;
        pl.rps = rps > (uint32_t)kMaxRps ? (uint32_t)kMaxRps : rps;
        pl.rows_max = rows;
        pl.plane_bytes = plane;
        pl.nbuf = nbuf;
        pl.tab_off = tab_off;
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

template <int KS, bool MASKED>
cudaError_t launch_ks(const UmmaParams& p, uint32_t smem, uint32_t grid, cudaStream_t s) {
  static bool attr_set = false;  // per instantiation, process-wide
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(umma_match_kernel<KS, MASKED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  umma_match_kernel<KS, MASKED><<<grid, kThreads, smem, s>>>(p);
  return cudaGetLastError();
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace

bool umma_supported(const MatchArgs& a) {
  Plan pl;
  if (a.precision == IPB_PRECISION_REFERENCE_F32) return false;
  if (a.mask && !a.mask_binary) return false;  // general u8 masks: CUDA-core byte planes
  return a.w >= 16 && a.h >= 8 && (size_t)a.w * a.h <= 33025 && make_plan(a.w, a.h, a.mask != nullptr, pl);
}

cudaError_t launch_umma(const MatchArgs& a, unsigned int* err_word, unsigned int tag) {
  Plan pl;
  const bool masked = a.mask != nullptr;
  if (!make_plan(a.w, a.h, masked, pl)) return cudaErrorNotSupported;
  UmmaParams p;
  p.img = a.img;
  p.W = a.W;
  p.H = a.H;
  p.tpl = a.tpl;
  p.mask = a.mask;
  p.w = a.w;
  p.h = a.h;
  p.kmma = pl.kmma;
  p.NT = pl.NT;
  p.rps = pl.rps;
  p.imgp = pl.imgp;
  p.rows_max = pl.rows_max;
  p.zrows = pl.zrows;
  p.zplane = pl.zplane;
  p.tab_off = pl.tab_off;
  p.z_off = pl.z_off;
  p.img_off = pl.img_off;
  p.rs_off = pl.rs_off;
  p.plane_bytes = pl.plane_bytes;
  p.nbuf = pl.nbuf;
  p.Wo = a.W - a.w + 1;
  p.Ho = a.H - a.h + 1;
  p.tiles_x = (p.Wo + kM - 1) / kM;
  p.tiles = p.tiles_x * ((p.Ho + pl.NT - 1) / pl.NT);
  p.method = a.method;
  p.precision = a.precision;
  const uintptr_t ia = reinterpret_cast<uintptr_t>(a.img);
  p.load_mode = ((ia & 15u) == 0 && (a.W & 15u) == 0) ? 2 : (((ia & 3u) == 0 && (a.W & 3u) == 0) ? 1 : 0);
  p.out = a.out;
  p.err = err_word;
  p.tag = tag;
  const uint32_t grid = p.tiles < (uint32_t)sm_count() ? p.tiles : (uint32_t)sm_count();
  cudaError_t e;
  timer_begin(a.timer, kKernelUmma, a.stream);
  if (masked) {
    switch (pl.ks) {
      case 8: e = launch_ks<8, true>(p, pl.smem, grid, a.stream); break;
      case 16: e = launch_ks<16, true>(p, pl.smem, grid, a.stream); break;
      default: e = launch_ks<32, true>(p, pl.smem, grid, a.stream); break;
    }
  } else {
    switch (pl.ks) {
      case 8: e = launch_ks<8, false>(p, pl.smem, grid, a.stream); break;
      case 16: e = launch_ks<16, false>(p, pl.smem, grid, a.stream); break;
      case 32: e = launch_ks<32, false>(p, pl.smem, grid, a.stream); break;
      default: e = launch_ks<64, false>(p, pl.smem, grid, a.stream); break;
    }
  }
  count_launch(kKernelUmma);
  timer_end(a.timer, a.stream);
  return e;
}

}  // namespace ipb
