// tm_umma.cu -- exact template matching on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, unsigned u8 x u8 -> s32, accumulators in tensor memory).
//
// Replaces the scalar walk of methods::*::score_at (src/template_matching.rs:
// 219-293, unmasked methods) for templates up to 256 x 128 pixels.
//
// Formulation. A CTA owns a tile of 128 output columns (x0 + m, m = tensor-
// memory lane) by NT output rows (y0 + n, n = tensor-memory column). For each
// image row r of the tile (r = 0 .. NT + h - 2, image row y0 + r):
//   A_r[m][k] = I[y0 + r][x0 + m + k]          (k < w; a Hankel row per lane)
//   B_r[n][k] = T[r - n][k]                     (0 <= r - n < h, else 0)
//   D[m][n]  += sum_k A_r[m][k] * B_r[n][k]
// so that after all rows D[m][n] = sum_{dy,dx} I[y0+n+dy][x0+m+dx] T[dy][dx],
// the exact cross-correlation X of that output. B_r is a window of one
// buffer Z (the template with its rows reversed and 16 zero rows on each
// side) stored in the canonical no-swizzle K-major layout, whose rows are
// 16 bytes apart: moving from r to r+1 moves B's start address by -16 bytes.
// Only the 16-aligned band of n where B_r is non-zero is issued (N = 16..NT).
//
// A_r goes straight into tensor memory: eight builder warps form each lane's
// K bytes from the staged image row with byte_perm and store them with
// tcgen05.st (the MMA reads A from tensor memory and only B from shared
// memory). The same words give the lane's row sum of squares with dp4a, from
// which the epilogue slides the window sum Y = sum I^2 over h rows, so SSE
// (Y - 2X + TSS) and the normalised methods need no integral image.
//
// Pipeline: builders fill 3 stages of RPS A rows; one thread issues the MMAs
// of a stage once it is full and commits the stage back to the builders;
// after the tile's last stage it commits the accumulator to the epilogue
// (the builder warps), which reads D with tcgen05.ld and writes the scores.
// Every wait is bounded (2 s); a wait that runs out sets the error word and
// the CTA leaves its loop, drains its MMAs and frees its tensor memory.
#include "tm_common.cuh"
#include "tm_internal.h"
#include "tm_sm100.cuh"

namespace ipb {
namespace {

using namespace sm100;

constexpr int kM = 128;
constexpr int kBuilderWarps = 8;
constexpr int kThreads = (kBuilderWarps + 1) * 32;
constexpr int kStages = 3;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr uint32_t kSmemHeader = 1024;
constexpr uint32_t kMinSmem = 120 * 1024;  // keeps residency at one CTA per SM

struct UmmaParams {
  const uint8_t* img;
  uint32_t W, H;
  const uint8_t* tplane;  // template plane 0 (T), rows of tpitch bytes, zero beyond w
  uint32_t tpitch, w, h;
  uint32_t kmma;   // K of the MMAs: w rounded up to 32
  uint32_t NT;     // output rows per tile (64 or 128)
  uint32_t rps;    // image rows per pipeline stage
  uint32_t imgp;   // staged image row pitch (bytes)
  uint32_t zrows;  // rows of the reversed-template buffer: h + 32
  uint32_t zbytes, imgbytes;
  const unsigned long long* tss;
  uint32_t Wo, Ho, tiles_x, tiles;
  int method, precision, vec16;
  float* out;
  unsigned int* err;
};

template <int KS>
__device__ __forceinline__ void build_row(const UmmaParams& p, const uint8_t* s_img, uint32_t r, uint32_t m,
                                          uint32_t taddr, uint32_t& rs_out) {
  const uint32_t* wp = reinterpret_cast<const uint32_t*>(s_img + r * p.imgp) + (m >> 2);
  const uint32_t sel = 0x3210u + (m & 3u) * 0x1111u;
  const uint32_t wq = p.w >> 2;  // full words inside the template width
  const uint32_t tail = (p.w & 3u) ? ((1u << (8u * (p.w & 3u))) - 1u) : 0u;
  uint32_t rs = 0;
  constexpr int CH = KS < 16 ? KS : 16;
#pragma unroll
  for (int c0 = 0; c0 < KS; c0 += CH) {
    uint32_t wv[CH + 1];
#pragma unroll
    for (int k = 0; k <= CH; ++k) wv[k] = wp[c0 + k];
    uint32_t a[CH];
#pragma unroll
    for (int k = 0; k < CH; ++k) a[k] = __byte_perm(wv[k], wv[k + 1], sel);
    if (c0 + CH <= (int)wq) {
#pragma unroll
      for (int k = 0; k < CH; ++k) rs = __dp4a(a[k], a[k], rs);
    } else {
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const uint32_t idx = c0 + k;
        const uint32_t mk = idx < wq ? 0xFFFFFFFFu : (idx == wq ? tail : 0u);
        const uint32_t v = a[k] & mk;
        rs = __dp4a(v, v, rs);
      }
    }
    if constexpr (CH == 16) {
      tmem_st16(taddr + c0, a);
    } else {
      tmem_st8(taddr + c0, a);
    }
  }
  rs_out = rs;
}

template <int KS>
__global__ void __launch_bounds__(kThreads, 1) umma_match_kernel(const UmmaParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  uint64_t* dfull = empty + kStages;
  uint64_t* drain = dfull + 1;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + 128);
  volatile int* s_err = reinterpret_cast<volatile int*>(smem + 132);
  uint8_t* zbuf = smem + kSmemHeader;
  uint8_t* s_img = zbuf + p.zbytes;
  uint32_t* s_rs = reinterpret_cast<uint32_t*>(s_img + p.imgbytes);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool mma_warp = warp == kBuilderWarps;
  const unsigned long long deadline0 = global_ns();
  (void)deadline0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], kBuilderWarps * 32);
      mbar_init(&empty[s], 1);
    }
    mbar_init(dfull, 1);
    mbar_init(drain, 1);
    *s_err = 0;
    mbar_init_fence();
  }
  if (mma_warp) {
    tmem_alloc(s_tmem, kTmemCols);
    tmem_relinquish();
  }
  // reversed template, K-chunk-major: chunk c holds rows j = 0..zrows-1 of 16 bytes,
  // row j = template row h-1-(j-16) for 16 <= j < h+16, zero otherwise
  {
    const uint32_t nchunks = p.kmma / 16;
    for (uint32_t idx = threadIdx.x; idx < nchunks * p.zrows; idx += kThreads) {
      const uint32_t c = idx / p.zrows, j = idx % p.zrows;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (j >= 16 && j < p.h + 16) {
        const uint32_t trow = p.h - 1 - (j - 16);
        v = *reinterpret_cast<const uint4*>(p.tplane + (size_t)trow * p.tpitch + 16 * c);
      }
      *reinterpret_cast<uint4*>(zbuf + (size_t)(c * p.zrows + j) * 16) = v;
    }
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t a_col0 = p.NT;
  const unsigned long long tss = *p.tss;
  const uint32_t zaddr = smem_u32(zbuf);
  const uint32_t chz = p.zrows * 16;

  uint32_t g = 0;        // pipeline stage fills so far (same count in builders and the MMA thread)
  uint32_t tcount = 0;   // tiles finished by this CTA
  bool ok = true;

  for (uint32_t tile = blockIdx.x; tile < p.tiles; tile += gridDim.x, ++tcount) {
    __syncthreads();
    if (*s_err) break;
    const uint32_t x0 = (tile % p.tiles_x) * kM;
    const uint32_t y0 = (tile / p.tiles_x) * p.NT;
    const uint32_t nrows = min(p.NT + p.h - 1, p.H - y0);
    // stage the tile's image rows, zero past the right edge
    {
      const uint8_t* src = p.img + (size_t)y0 * p.W;
      const uint32_t chunks = p.imgp / 16;
      for (uint32_t idx = threadIdx.x; idx < nrows * chunks; idx += kThreads) {
        const uint32_t r = idx / chunks, c = (idx % chunks) * 16;
        const uint32_t gx = x0 + c;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        const uint8_t* row = src + (size_t)r * p.W;
        if (p.vec16 && gx + 16 <= p.W) {
          v = __ldg(reinterpret_cast<const uint4*>(row + gx));
        } else if (gx < p.W) {
          uint32_t wd[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (gx + k < p.W) wd[k >> 2] |= (uint32_t)__ldg(row + gx + k) << (8 * (k & 3));
          v = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        }
        *reinterpret_cast<uint4*>(s_img + r * p.imgp + c) = v;
      }
    }
    __syncthreads();
    if (*s_err) break;
    const uint32_t nst = (nrows + p.rps - 1) / p.rps;
    const unsigned long long deadline = global_ns() + kWaitNs;

    if (!mma_warp) {
      const uint32_t q = warp & 3, half = warp >> 2;
      const uint32_t m = q * 32 + lane;
      const uint32_t lane_base = q * 32;
      // zero this warp's share of the accumulator (lanes of quadrant q, half of the columns)
      {
        const uint32_t zero16[16] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        for (uint32_t c = half * (p.NT / 2); c < (half + 1) * (p.NT / 2); c += 16)
          tmem_st16(tmem_addr(tmem, lane_base, c), zero16);
      }
      for (uint32_t st = 0; st < nst; ++st, ++g) {
        const uint32_t s = g % kStages;
        if (g >= kStages && !mbar_wait(&empty[s], ((g / kStages) + 1) & 1u, deadline)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t r_end = min(nrows, (st + 1) * p.rps);
        for (uint32_t r = st * p.rps + half; r < r_end; r += 2) {
          const uint32_t slot = r - st * p.rps;
          uint32_t rs;
          build_row<KS>(p, s_img, r, m, tmem_addr(tmem, lane_base, a_col0 + (s * p.rps + slot) * KS), rs);
          s_rs[r * kM + m] = rs;
        }
        tmem_wait_st();
        tc_fence_before();
        mbar_arrive(&full[s]);
      }
      if (ok && !mbar_wait(dfull, tcount & 1u, deadline)) ok = false;
      // all 256 builder threads reach this (every wait above is bounded): the
      // row sums written by the other builder warps are visible after it
      asm volatile("bar.sync 1, 256;" ::: "memory");
      if (ok) {
        tc_fence_after();
        // epilogue: this warp's lanes (output columns) x half of the rows
        const uint32_t x = x0 + m;
        const uint32_t n_begin = half * (p.NT / 2), n_end = n_begin + p.NT / 2;
        unsigned long long Y = 0;
        for (uint32_t r = n_begin; r < n_begin + p.h; ++r) Y += r < nrows ? s_rs[r * kM + m] : 0u;
        for (uint32_t n0 = n_begin; n0 < n_end; n0 += 32) {
          uint32_t v[32];
          tmem_ld32(tmem_addr(tmem, lane_base, n0), v);
          tmem_wait_ld();
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const uint32_t n = n0 + k;
            const uint32_t y = y0 + n;
            if (x < p.Wo && y < p.Ho)
              p.out[(size_t)y * p.Wo + x] = finish_score(p.method, p.precision, v[k], Y, tss);
            const uint32_t ra = n + p.h, rb = n;
            Y += (ra < nrows ? s_rs[ra * kM + m] : 0u);
            Y -= (rb < nrows ? s_rs[rb * kM + m] : 0u);
          }
        }
      }
      if (!ok) {
        *s_err = 1;
        atomicOr(p.err, 1u);
      }
    } else {
      if (lane == 0) {
        for (uint32_t st = 0; st < nst; ++st, ++g) {
          const uint32_t s = g % kStages;
          if (!mbar_wait(&full[s], (g / kStages) & 1u, deadline)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t r_end = min(nrows, (st + 1) * p.rps);
          for (uint32_t r = st * p.rps; r < r_end; ++r) {
            // output rows n with 0 <= r - n < h, inside the tile and the map
            const uint32_t lo = r + 1 > p.h ? r + 1 - p.h : 0u;
            uint32_t hi = min(p.NT - 1, r);
            hi = min(hi, p.Ho - 1 - y0);
            if (lo > hi) continue;
            const uint32_t n0 = lo & ~15u, n1 = (hi + 16u) & ~15u;
            const uint32_t j0 = n0 + p.h + 15u - r;  // first Z row of this band
            const uint32_t idesc = idesc_u8u8_s32(kM, n1 - n0);
            const uint32_t a = tmem_addr(tmem, 0, a_col0 + (s * p.rps + (r - st * p.rps)) * KS);
            for (uint32_t kk = 0; kk < p.kmma / 32; ++kk) {
              const uint64_t bdesc = smem_desc_noswizzle(zaddr + (2 * kk) * chz + j0 * 16, chz, 128);
              mma_i8_ts(tmem_addr(tmem, 0, n0), a + kk * 8, bdesc, idesc, 1u);
            }
          }
          mma_commit(&empty[s]);
        }
        if (ok) mma_commit(dfull);
        if (!ok) {
          *s_err = 1;
          atomicOr(p.err, 1u);
        }
      }
      __syncwarp();
    }
  }

  // drain outstanding MMAs, then free tensor memory
  __syncthreads();
  if (mma_warp) {
    if (lane == 0) {
      mma_commit(drain);
      if (!mbar_wait(drain, 0, global_ns() + kWaitNs)) atomicOr(p.err, 2u);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

struct Plan {
  uint32_t kmma, ks, NT, rps, imgp, zrows, zbytes, imgbytes, smem;
};

bool make_plan(uint32_t w, uint32_t h, Plan& pl) {
  if (w < 8 || w > 256 || h < 1 || h > 128) return false;
  pl.kmma = (w + 31) & ~31u;
  uint32_t ks = 8;
  while (ks * 4 < pl.kmma) ks *= 2;
  pl.ks = ks;
  pl.imgp = kM + 4 * ks + 16;
  pl.zrows = h + 32;
  pl.zbytes = (pl.kmma / 16) * pl.zrows * 16;
  for (uint32_t nt : {128u, 64u}) {
    const uint32_t rows = nt + h - 1;
    const uint32_t imgbytes = (uint32_t)align_up((size_t)rows * pl.imgp, 128);
    const uint32_t smem = kSmemHeader + (uint32_t)align_up(pl.zbytes, 128) + imgbytes + rows * kM * 4;
    // tensor memory: NT accumulator columns + kStages * rps A rows of ks columns
    const uint32_t rps = (kTmemCols - nt) / (kStages * ks);
    if (smem <= 227u * 1024u && rps >= 2) {
      pl.NT = nt;
      pl.rps = rps > 16 ? 16 : rps & ~1u;
      pl.zbytes = (uint32_t)align_up(pl.zbytes, 128);
      pl.imgbytes = imgbytes;
      pl.smem = smem < kMinSmem ? kMinSmem : smem;
      return true;
    }
  }
  return false;
}

template <int KS>
cudaError_t launch_ks(const UmmaParams& p, uint32_t smem, uint32_t grid, cudaStream_t s) {
  static bool attr_set = false;  // per instantiation, process-wide
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(umma_match_kernel<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  umma_match_kernel<KS><<<grid, kThreads, smem, s>>>(p);
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
  return !a.mask && a.precision != IPB_PRECISION_REFERENCE_F32 && a.w >= 16 && a.h >= 8 &&
         (size_t)a.w * a.h <= 33025 && make_plan(a.w, a.h, pl);
}

size_t umma_scratch_bytes(const MatchArgs& a) { return prep_scratch_bytes(a); }

cudaError_t launch_umma(const MatchArgs& a, void* scratch) {
  Plan pl;
  if (!make_plan(a.w, a.h, pl)) return cudaErrorNotSupported;
  uint8_t* base = static_cast<uint8_t*>(scratch);
  const size_t planes_bytes = prep_scratch_bytes(a) - 256;
  unsigned long long* tss = reinterpret_cast<unsigned long long*>(base + planes_bytes);
  unsigned int* err = reinterpret_cast<unsigned int*>(base + planes_bytes + 8);
  cudaError_t e = launch_prep(a, base, tss);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(err, 0, sizeof(unsigned int), a.stream);
  if (e != cudaSuccess) return e;

  UmmaParams p;
  p.img = a.img;
  p.W = a.W;
  p.H = a.H;
  p.tplane = base;
  p.tpitch = (uint32_t)template_pitch(a.w);
  p.w = a.w;
  p.h = a.h;
  p.kmma = pl.kmma;
  p.NT = pl.NT;
  p.rps = pl.rps;
  p.imgp = pl.imgp;
  p.zrows = pl.zrows;
  p.zbytes = pl.zbytes;
  p.imgbytes = pl.imgbytes;
  p.tss = tss;
  p.Wo = a.W - a.w + 1;
  p.Ho = a.H - a.h + 1;
  p.tiles_x = (p.Wo + kM - 1) / kM;
  p.tiles = p.tiles_x * ((p.Ho + pl.NT - 1) / pl.NT);
  p.method = a.method;
  p.precision = a.precision;
  p.vec16 = ((reinterpret_cast<uintptr_t>(a.img) & 15u) == 0 && (a.W & 15u) == 0) ? 1 : 0;
  p.out = a.out;
  p.err = err;
  const uint32_t grid = p.tiles < (uint32_t)sm_count() ? p.tiles : (uint32_t)sm_count();
  timer_begin(a.timer, kKernelUmma, a.stream);
  switch (pl.ks) {
    case 8: e = launch_ks<8>(p, pl.smem, grid, a.stream); break;
    case 16: e = launch_ks<16>(p, pl.smem, grid, a.stream); break;
    case 32: e = launch_ks<32>(p, pl.smem, grid, a.stream); break;
    default: e = launch_ks<64>(p, pl.smem, grid, a.stream); break;
  }
  count_launch(kKernelUmma);
  timer_end(a.timer, a.stream);
  return e;
}

unsigned int* umma_error_word(void* scratch, const MatchArgs& a) {
  return reinterpret_cast<unsigned int*>(static_cast<uint8_t*>(scratch) + prep_scratch_bytes(a) - 256 + 8);
}

}  // namespace ipb
