// tm_many.cu -- many templates of one size against one image on tcgen05.
//
// The reference scores one template per call (match_template,
// src/template_matching.rs:78-92). For a bank of templates the work becomes
// one GEMM per output column x:
//   D[m][t] = sum_{dy,dx} I[y0 + m + dy][x + dx] * T_t[dy][dx]
// over 128 consecutive output rows m, a block of templates t and
// K = the template's pixels in (dy, dx) order, 32 bytes per MMA step.
//
// Image operand: a "strip" of the image for column x -- for each 16-byte
// column chunk j, the rows y0 .. y0 + 127 + h - 1 of bytes [x + 16j,
// x + 16j + 16), stored 16 bytes per row in the canonical no-swizzle K-major
// layout. The operand for template row dy is the same strip started dy rows
// (16*dy bytes) later, so one strip (about 5 KB) serves all h template rows.
// Template operand: the template block, K-major, resident in shared memory
// for the CTA's lifetime.
//
// Two operand assignments:
//  * templates as M (kTplM): A = 128 templates, B = the strip (N = 128
//    positions). Tensor-memory lanes are templates, so each epilogue store
//    instruction writes 32 consecutive templates of one position -- a full
//    128-byte line of the position-major output -- and every lane keeps its
//    template's extremes in registers. Used when a block of 128 templates
//    fits in shared memory (h * round32(w) <= about 1200 bytes).
//  * positions as M: A = the strip (M = 128 positions), B = NB templates
//    (a multiple of 16, at most 112), for larger templates.
//
// Roles: all warps stage each image tile (cp.async) and compute the window
// sums Y = sum I^2 of its positions; then 2 builder warps build strips, one
// warp issues the MMAs (one flat loop, one elected lane) and 16 epilogue
// warps (four per tensor-memory lane quadrant) read the accumulator
// (double-buffered in tensor memory), apply the method, write the scores and
// fold them into per-template extremes. Scores are position-major:
// out[(y * Wo + x) * n_templates + t].
// Every wait is bounded (2 s) and reports through the error word.
#include <type_traits>

#include "tm_common.cuh"
#include "tm_internal.h"
#include "tm_sm100.cuh"

namespace ipb {
namespace {

using namespace sm100;

constexpr int kM = 128;           // output rows per tile
constexpr int kXT = 32;           // output columns per tile
constexpr int kBuildWarps = 2;
constexpr int kEpiWarps = 16;  // four per lane quadrant: the epilogue is the longest role
constexpr int kMmaWarp = kBuildWarps + kEpiWarps;
constexpr int kEpiPerQuad = kEpiWarps / 4;      // epilogue warps per tensor-memory lane quadrant
constexpr int kPosW = kM / kEpiPerQuad;         // templates as M: positions per epilogue warp
constexpr int kThreads = (kMmaWarp + 1) * 32;
constexpr int kStrips = 3;
constexpr uint32_t kTmemCols = 256;  // two accumulators of up to 128 columns
constexpr unsigned long long kWaitNs = kDefaultWaitNs;  // the final drain's budget

struct ManyParams {
  const uint8_t* img;
  uint32_t W, H;
  const uint8_t* tpl;  // n templates of w x h, contiguous
  uint32_t w, h, n;
  uint32_t kw;       // w rounded up to 32
  uint32_t NB;       // templates per block: 128 (templates as M) or a multiple of 16
  uint32_t nblocks;  // ceil(n / NB)
  uint32_t Wo, Ho, bands, xtiles, spatial;  // spatial tiles = bands * xtiles
  uint32_t rows;     // strip rows: 128 + h - 1
  uint32_t ip;       // staged image row pitch
  uint32_t b_off, tss_off, img_off, strip_off, y_off, v_off, ext_off, ry_off;
  int method, precision, vec4;  // vec4: 16-byte score stores (positions as M)
  int img16;                    // image rows 16-byte aligned: cp.async staging
  float* out;                 // may be null (extremes only)
  unsigned long long* ext;    // 2 keys per template or null
  unsigned int* err;
  unsigned int tag;
  unsigned long long wait_ns;  // budget of the bounded waits per tile (pipeline_wait_ns())
  uint32_t stall;              // pipeline_stall() at launch
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t order_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// State of an epilogue warp for one tile.
struct EpiCtx {
  const ManyParams* p;
  uint32_t tmem;
  uint64_t* dfull;
  uint64_t* dempty;
  const uint32_t* s_y;
  const uint32_t* s_tss;
  unsigned long long* s_ext;
  double* s_ry;  // [kEpiWarps][kPosW] reciprocal roots of the strip's Y (templates as M)
  uint32_t gx, nx, x0, y0, t0, nt;
  uint32_t e;  // epilogue warp index: lane quadrant (e + kBuildWarps) & 3, share e >> 2
  uint32_t lane;
  unsigned long long deadline;
  unsigned long long kmin, kmax;  // templates as M: this lane's running extremes keys
};

// Drains the tile's accumulators with the method and precision fixed at
// compile time, so the 16 scores of a tensor-memory load are independent
// straight-line code. Returns false when a wait ran out.
template <bool kTplM, int kMethod, int kPrec, bool kExt>
__device__ __forceinline__ bool epilogue(EpiCtx& c) {
  const ManyParams& p = *c.p;
  const uint32_t q = (c.e + kBuildWarps) & 3;  // = warp & 3, the lanes this warp may access
  if constexpr (kTplM) {
    // lanes are templates; this warp takes kPosW (= 32) of the tile's 128
    // positions, as two halves of 16 (one tensor-memory load each)
    static_assert(kPosW == 32, "two halves of 16 positions per strip");
    const uint32_t mb = (c.e >> 2) * kPosW;
    const uint32_t tl = q * 32 + c.lane;
    const bool t_ok = tl < c.nt;
    const uint32_t tss = c.s_tss[tl];
    // EXACT_FP64 normalisation: 1/sqrt(Y) once per position (shared by the
    // warp's 32 templates) and 1/sqrt(T) once per lane
    constexpr bool kNormW = method_is_norm(kMethod) && kPrec == IPB_PRECISION_EXACT_FP64;
    double* s_ryw = c.s_ry + c.e * kPosW;
    const double rT = (kNormW && tss) ? rsqrt_u32(tss) : 0.0;
    const int mvalid = (int)p.Ho - (int)(c.y0 + mb);  // positions of the share inside the map
    const size_t rstride = (size_t)p.Wo * p.n;
    auto score_of = [&](uint32_t v, uint32_t y) -> uint32_t {
      return method_is_sse(kMethod) ? (y + tss - 2u * v) : v;
    };
    for (uint32_t xi = 0; xi < c.nx; ++xi) {
      const uint32_t g = c.gx + xi, d = g & 1u;
      if (!__all_sync(0xffffffffu, mbar_wait_sleep(&c.dfull[d], (g >> 1) & 1u, c.deadline))) return false;
      tc_fence_after();
      const uint32_t x = c.x0 + xi;
      const uint32_t* ycol = c.s_y + xi * kM + mb;
      float* ocol = (p.out && t_ok) ? p.out + ((size_t)(c.y0 + mb) * p.Wo + x) * p.n + c.t0 + tl : nullptr;
      // a zero norm anywhere in the share (a window of zeros, or this lane's
      // template all zeros) sends the strip through the general quotient
      bool general = false;
      if constexpr (kNormW) {
        __syncwarp();
        const uint32_t yv = ycol[c.lane];
        s_ryw[c.lane] = yv ? rsqrt_u32(yv) : 0.0;
        general = __any_sync(0xffffffffu, yv == 0u) || rT == 0.0;
        __syncwarp();
      }
#pragma unroll
      for (int half = 0; half < 32; half += 16) {
        if (half >= mvalid) break;  // warp-uniform: past the map's last row
        const int nv = min(16, mvalid - half);
        const uint32_t taddr = tmem_addr(c.tmem, q * 32, d * 128 + mb + half);
        float* o = ocol ? ocol + (size_t)half * rstride : nullptr;
        // Fast pass: each value is scored branch-free, stored at once and
        // folded into the half's smallest and largest bits (scores are never
        // negative, so f32 bits order like the values). FP64 quotients near
        // an f32 rounding midpoint are flagged.
        uint32_t b[16];
        uint32_t mn = 0xFFFFFFFFu, mx = 0u;
        bool undecided = false;
        {
          uint32_t v[16], Y[16];
          tmem_ld16(taddr, v);
#pragma unroll
          for (int k = 0; k < 16; k += 4) {
            const uint4 y4 = *reinterpret_cast<const uint4*>(ycol + half + k);
            Y[k] = y4.x;
            Y[k + 1] = y4.y;
            Y[k + 2] = y4.z;
            Y[k + 3] = y4.w;
          }
          tmem_wait_ld();
          auto pass = [&](auto full_tag) {
            constexpr bool kFull = decltype(full_tag)::value;
#pragma unroll
            for (int k = 0; k < 16; k += 2) {
              if constexpr (kNormW) {
                const double2 r2 = *reinterpret_cast<const double2*>(s_ryw + half + k);
                b[k] = norm_bits_fp64_fast(score_of(v[k], Y[k]), __dmul_rn(r2.x, rT), undecided);
                b[k + 1] = norm_bits_fp64_fast(score_of(v[k + 1], Y[k + 1]), __dmul_rn(r2.y, rT), undecided);
              } else {
                b[k] = __float_as_uint(finish_score32(kMethod, kPrec, v[k], Y[k], tss));
                b[k + 1] = __float_as_uint(finish_score32(kMethod, kPrec, v[k + 1], Y[k + 1], tss));
              }
#pragma unroll
              for (int u = 0; u < 2; ++u)
                if (kFull || k + u < nv) {
                  if (o) o[(size_t)(k + u) * rstride] = __uint_as_float(b[k + u]);
                  mn = min(mn, b[k + u]);
                  mx = max(mx, b[k + u]);
                }
            }
          };
          if (nv == 16)
            pass(std::true_type{});
          else
            pass(std::false_type{});
        }
        // Rare and warp-uniform: a half with a flagged or zero-norm quotient
        // reloads its sums, re-scores the flagged values through the general
        // quotient, stores them again and recomputes the half's extremes.
        if (__any_sync(0xffffffffu, general || undecided)) {
          uint32_t v[16];
          tmem_ld16(taddr, v);
          tmem_wait_ld();
          if constexpr (kNormW) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              if (k >= nv) break;
              const uint32_t yk = ycol[half + k];
              const uint32_t sk = score_of(v[k], yk);
              const double w = __dmul_rn(s_ryw[half + k], rT);
              bool u = general;
              if (!general) norm_bits_fp64_fast(sk, w, u);
              if (u) {
                b[k] = __float_as_uint(norm_quotient_fp64_w(sk, w, yk, tss));
                if (o) o[(size_t)k * rstride] = __uint_as_float(b[k]);
              }
            }
          }
          mn = 0xFFFFFFFFu;
          mx = 0u;
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (k < nv) {
              mn = min(mn, b[k]);
              mx = max(mx, b[k]);
            }
        }
        if constexpr (kExt) {
          // the half's extremes reach this lane's running keys only when the
          // key with the half's first index does (the 16 positions are rows of
          // one column: the lowest k is the lowest index); then the first
          // occurrence is found in this lane alone
          const uint32_t idx0 = (c.y0 + mb + half) * p.Wo + x;
          if (t_ok && ((((unsigned long long)(mn | 0x80000000u) << 32) | idx0) < c.kmin)) {
            uint32_t j = 0;
#pragma unroll
            for (int k = 15; k >= 0; --k)
              if (b[k] == mn) j = k;
            c.kmin = min(c.kmin, ((unsigned long long)(mn | 0x80000000u) << 32) | (idx0 + j * p.Wo));
          }
          if (t_ok && ((((unsigned long long)(mx | 0x80000000u) << 32) | (0xFFFFFFFFu - idx0)) > c.kmax)) {
            uint32_t j = 0;
#pragma unroll
            for (int k = 15; k >= 0; --k)
              if (b[k] == mx) j = k;
            c.kmax = max(c.kmax, ((unsigned long long)(mx | 0x80000000u) << 32) | (0xFFFFFFFFu - (idx0 + j * p.Wo)));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (c.lane == 0) mbar_arrive(&c.dempty[d]);
    }
    return true;
  } else {
    // lanes are positions (rows); the quadrant's warps take the block's
    // 16-template chunks in turn
    const uint32_t m = q * 32 + c.lane, y = c.y0 + m;
    const bool row_ok = y < p.Ho;
    for (uint32_t xi = 0; xi < c.nx; ++xi) {
      const uint32_t g = c.gx + xi, d = g & 1u;
      if (!__all_sync(0xffffffffu, mbar_wait_sleep(&c.dfull[d], (g >> 1) & 1u, c.deadline))) return false;
      tc_fence_after();
      const uint32_t x = c.x0 + xi;
      const uint32_t Y = c.s_y[xi * kM + m];
      float* orow = p.out ? p.out + ((size_t)y * p.Wo + x) * p.n + c.t0 : nullptr;
      for (uint32_t cc = (c.e >> 2) * 16; cc < p.NB; cc += 16 * kEpiPerQuad) {
        uint32_t v[16];
        tmem_ld16(tmem_addr(c.tmem, q * 32, d * 128 + cc), v);
        tmem_wait_ld();
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) f[k] = finish_score32(kMethod, kPrec, v[k], Y, c.s_tss[cc + k]);
        if (orow && row_ok) {
          if (p.vec4 && cc + 16 <= c.nt) {
#pragma unroll
            for (int k = 0; k < 16; k += 4)
              *reinterpret_cast<float4*>(orow + cc + k) = make_float4(f[k], f[k + 1], f[k + 2], f[k + 3]);
          } else {
            for (int k = 0; k < 16; ++k)
              if (cc + k < c.nt) orow[cc + k] = f[k];
          }
        }
        if constexpr (kExt) {
          // per template: smallest / largest value over this warp's 32 rows,
          // the lowest row (= lowest linear index at this x) among ties;
          // lane k keeps template cc + k's result
          uint32_t my_mn = 0xFFFFFFFFu, my_ln = 0, my_mx = 0, my_lx = 0;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const uint32_t key = row_ok ? order_key(f[k]) : 0xFFFFFFFFu;
            const uint32_t kmn = __reduce_min_sync(0xffffffffu, key);
            const uint32_t ln = __ffs(__ballot_sync(0xffffffffu, key == kmn)) - 1;
            const uint32_t keyx = row_ok ? order_key(f[k]) : 0u;
            const uint32_t kmx = __reduce_max_sync(0xffffffffu, keyx);
            const uint32_t lx = __ffs(__ballot_sync(0xffffffffu, keyx == kmx)) - 1;
            if (c.lane == (uint32_t)k) {
              my_mn = kmn;
              my_ln = ln;
              my_mx = kmx;
              my_lx = lx;
            }
          }
          if (c.lane < 16 && cc + c.lane < c.nt) {
            const uint32_t ymn = c.y0 + q * 32 + my_ln, ymx = c.y0 + q * 32 + my_lx;
            if (ymn < p.Ho)
              atomicMin(&c.s_ext[2 * (cc + c.lane)], ((unsigned long long)my_mn << 32) | (ymn * p.Wo + x));
            if (ymx < p.Ho)
              atomicMax(&c.s_ext[2 * (cc + c.lane) + 1],
                        ((unsigned long long)my_mx << 32) | (0xFFFFFFFFu - (ymx * p.Wo + x)));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (c.lane == 0) mbar_arrive(&c.dempty[d]);
    }
    return true;
  }
}

// One kernel per (operand assignment, method, precision, extremes): each
// gets its own register allocation for its epilogue. Precision only affects
// the normalised methods; the others use EXACT_FP64's instance.
template <bool kTplM, int kMethod, int kPrec, bool kExt>
__global__ void __launch_bounds__(kThreads, 1) many_match_kernel(const __grid_constant__ ManyParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* sfull = reinterpret_cast<uint64_t*>(smem);   // [kStrips] strip built
  uint64_t* sempty = sfull + kStrips;                    // [kStrips] strip consumed by the MMAs
  uint64_t* dfull = sempty + kStrips;                    // [2] accumulator ready
  uint64_t* dempty = dfull + 2;                          // [2] accumulator drained
  uint64_t* drain = dempty + 2;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + 128);
  volatile int* s_err = reinterpret_cast<volatile int*>(smem + 132);
  uint8_t* bmat = smem + p.b_off;                        // templates, K-major chunks
  uint32_t* s_tss = reinterpret_cast<uint32_t*>(smem + p.tss_off);
  uint8_t* s_img = smem + p.img_off;
  uint8_t* s_strip = smem + p.strip_off;
  uint32_t* s_y = reinterpret_cast<uint32_t*>(smem + p.y_off);   // [kXT][kM]
  uint32_t* s_v = reinterpret_cast<uint32_t*>(smem + p.v_off);   // [rows][kXT]
  unsigned long long* s_ext = reinterpret_cast<unsigned long long*>(smem + p.ext_off);  // [NB][2]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t nch = p.kw / 16;
  const uint32_t strip_bytes = nch * p.rows * 16;
  const uint32_t tb = blockIdx.x % p.nblocks;              // this CTA's template block
  const uint32_t t0 = tb * p.NB;
  const uint32_t nt = min(p.NB, p.n - t0);                 // templates in the block

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStrips; ++s) {
      mbar_init(&sfull[s], kBuildWarps);  // one arrive per builder warp
      mbar_init(&sempty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      mbar_init(&dfull[d], 1);
      mbar_init(&dempty[d], kEpiWarps);   // one arrive per epilogue warp
    }
    mbar_init(drain, 1);
    *s_err = 0;
    mbar_init_fence();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(s_tmem, kTmemCols);
    tmem_relinquish();
  }
  // template block: chunk (dy, j) holds NB rows of 16 bytes (template t's
  // bytes [16j, 16j+16) of row dy; zero past w and for absent templates)
  for (uint32_t idx = threadIdx.x; idx < p.h * nch * p.NB; idx += kThreads) {
    const uint32_t t = idx % p.NB, c = idx / p.NB;  // c = dy * nch + j
    const uint32_t dy = c / nch, j = c % nch;
    uint32_t wd[4] = {0u, 0u, 0u, 0u};
    if (t < nt) {
      const uint8_t* row = p.tpl + ((size_t)(t0 + t) * p.h + dy) * p.w;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t dx = 16 * j + k;
        if (dx < p.w) wd[k >> 2] |= (uint32_t)__ldg(row + dx) << (8 * (k & 3));
      }
    }
    *reinterpret_cast<uint4*>(bmat + (size_t)c * p.NB * 16 + t * 16) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
  }
  // template constants TSS_t = sum T_t^2 (< 2^32 for templates up to 64 x 64)
  for (uint32_t t = warp; t < p.NB; t += kThreads / 32) {
    uint32_t s = 0;
    if (t < nt)
      for (uint32_t k = lane; k < p.w * p.h; k += 32) {
        const uint32_t v = __ldg(p.tpl + (size_t)(t0 + t) * p.w * p.h + k);
        s += v * v;
      }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) s_tss[t] = s;
  }
  for (uint32_t i = threadIdx.x; i < 2 * p.NB; i += kThreads) s_ext[i] = (i & 1) ? 0ull : ~0ull;
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t idesc = kTplM ? idesc_u8u8_s32(128, kM) : idesc_u8u8_s32(kM, p.NB);
  constexpr bool do_ext = kExt;
  // templates as M: this lane's template and its running extremes keys
  const uint32_t tl = ((uint32_t)warp & 3u) * 32 + lane;
  const bool t_ok = tl < nt;
  unsigned long long kmin = ~0ull, kmax = 0ull;

  uint32_t gx = 0;  // strips built / consumed so far (global x counter, same in all roles)
  bool ok = true;
  const uint32_t cta_in_block = blockIdx.x / p.nblocks;
  const uint32_t ctas_per_block = gridDim.x / p.nblocks;

  for (uint32_t sp = cta_in_block; sp < p.spatial; sp += ctas_per_block) {
    __syncthreads();
    if (*s_err) break;
    const uint32_t y0 = (sp / p.xtiles) * kM, x0 = (sp % p.xtiles) * kXT;
    const uint32_t nrows = min(p.rows, p.H - y0);
    const uint32_t nx = min((uint32_t)kXT, p.Wo - x0);
    // stage the tile's image rows (all threads), zero past the right edge
    {
      const uint32_t chunks = p.ip / 16;
      const uint8_t* src = p.img + (size_t)y0 * p.W;
      for (uint32_t idx = threadIdx.x; idx < nrows * chunks; idx += kThreads) {
        const uint32_t r = idx / chunks, c = (idx % chunks) * 16, gxx = x0 + c;
        uint8_t* dst = s_img + r * p.ip + c;
        if (p.img16 && gxx + 16 <= p.W) {
          cp_async16(smem_u32(dst), src + (size_t)r * p.W + gxx, 16);
        } else {
          uint32_t wd[4] = {0u, 0u, 0u, 0u};
          for (int k = 0; k < 16; ++k)
            if (gxx + k < p.W) wd[k >> 2] |= (uint32_t)__ldg(src + (size_t)r * p.W + gxx + k) << (8 * (k & 3));
          *reinterpret_cast<uint4*>(dst) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        }
      }
      cp_async_commit();
      cp_async_wait_all();
    }
    __syncthreads();
    // window sums of I^2 for the tile's positions: V = row sums over w, then Y over h
    for (uint32_t r = threadIdx.x; r < nrows; r += kThreads) {
      const uint8_t* row = s_img + r * p.ip;
      uint32_t s = 0;
      for (uint32_t dx = 0; dx < p.w; ++dx) s += (uint32_t)row[dx] * row[dx];
      for (uint32_t xi = 0; xi < (uint32_t)kXT; ++xi) {
        s_v[r * kXT + xi] = s;
        const uint32_t a = row[xi + p.w], b = row[xi];
        s += a * a - b * b;
      }
    }
    __syncthreads();
    for (uint32_t idx = threadIdx.x; idx < (uint32_t)kXT * (kM / 32); idx += kThreads) {
      const uint32_t xi = idx % kXT, m0 = (idx / kXT) * 32;
      uint32_t s = 0;
      for (uint32_t dy = 0; dy < p.h; ++dy) s += (m0 + dy < nrows) ? s_v[(m0 + dy) * kXT + xi] : 0u;
      for (uint32_t m = m0; m < m0 + 32; ++m) {
        s_y[xi * kM + m] = s;
        const uint32_t a = (m + p.h < nrows) ? s_v[(m + p.h) * kXT + xi] : 0u;
        const uint32_t b = (m < nrows) ? s_v[m * kXT + xi] : 0u;
        s += a - b;
      }
    }
    __syncthreads();
    const unsigned long long deadline = global_ns() + p.wait_ns;

    if (warp < kBuildWarps) {
      // strips: S_x[j][rho] = image row rho, bytes [xi + 16j, xi + 16j + 16)
      for (uint32_t xi = 0; xi < nx; ++xi) {
        const uint32_t g = gx + xi, s = g % kStrips;
        const bool got = g < kStrips || mbar_wait_sleep(&sempty[s], ((g / kStrips) + 1) & 1u, deadline);
        if (!__all_sync(0xffffffffu, got)) {  // warp-uniform: the warp arrives as one below
          ok = false;
          break;
        }
        uint8_t* strip = s_strip + s * strip_bytes;
        const uint32_t sel = 0x3210u + (xi & 3u) * 0x1111u;
        for (uint32_t idx = threadIdx.x; idx < nch * nrows; idx += kBuildWarps * 32) {
          const uint32_t j = idx / nrows, r = idx % nrows;
          const uint32_t* wp = reinterpret_cast<const uint32_t*>(s_img + r * p.ip) + (xi >> 2) + 4 * j;
          const uint32_t w0 = wp[0], w1 = wp[1], w2 = wp[2], w3 = wp[3], w4 = wp[4];
          *reinterpret_cast<uint4*>(strip + (j * p.rows + r) * 16) =
              make_uint4(__byte_perm(w0, w1, sel), __byte_perm(w1, w2, sel), __byte_perm(w2, w3, sel),
                         __byte_perm(w3, w4, sel));
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sfull[s]);
      }
      if (!ok) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    } else if (warp == kMmaWarp) {
      // warp-uniform issue loop: descriptors advance by adding to their
      // 16-byte-unit start-address field (shared addresses stay below 2^18)
      const uint32_t lbo_s = p.rows * 16, lbo_t = p.NB * 16;
      const uint32_t sstep = lbo_s >> 4, tstep = lbo_t >> 4;
      const uint64_t tdesc0 = smem_desc_noswizzle(smem_u32(bmat), lbo_t, 128);
      const uint32_t nk = p.kw / 32;
      // test hook: a wait on the drain barrier, which nothing arrives at before the end
      if (p.stall && !__all_sync(0xffffffffu, mbar_wait(drain, 0, deadline))) ok = false;
      for (uint32_t xi = 0; ok && xi < nx; ++xi) {
        const uint32_t g = gx + xi, s = g % kStrips, d = g & 1u;
        const bool got_s = mbar_wait(&sfull[s], (g / kStrips) & 1u, deadline);
        const bool got_d = got_s && (g < 2 || mbar_wait(&dempty[d], ((g >> 1) + 1) & 1u, deadline));
        if (!__all_sync(0xffffffffu, got_s && got_d)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dt = tmem + d * 128;
        // one flat loop over template rows with running descriptors: the
        // strip advances one 16-byte row per template row, the template block
        // one row of nch chunks (a nested loop with computed descriptors
        // issued at under half the tensor pipe's rate)
        uint64_t sd = smem_desc_noswizzle(smem_u32(s_strip + s * strip_bytes), lbo_s, 128);
        uint64_t td = tdesc0;
        const uint64_t tdy = (uint64_t)(nch * tstep);
        auto mma = [&](uint64_t tdk, uint64_t sdk, uint32_t acc) {
          if constexpr (kTplM)
            mma_i8_ss_warp(dt, tdk, sdk, idesc, acc);
          else
            mma_i8_ss_warp(dt, sdk, tdk, idesc, acc);
        };
        if (nk == 1) {
          for (uint32_t dy = 0; dy < p.h; ++dy, sd += 1, td += tdy) mma(td, sd, dy != 0);
        } else {  // two 32-byte K steps per template row (w in 33..64)
          for (uint32_t dy = 0; dy < p.h; ++dy, sd += 1, td += tdy) {
            mma(td, sd, dy != 0);
            mma(td + 2 * tstep, sd + 2 * sstep, 1u);
          }
        }
        mma_commit_warp(&sempty[s]);
        mma_commit_warp(&dfull[d]);
      }
      if (!ok && lane == 0) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    } else {
      EpiCtx c{&p, tmem, dfull, dempty, s_y, s_tss, s_ext, reinterpret_cast<double*>(smem + p.ry_off),
               gx, nx, x0, y0, t0, nt,
               (uint32_t)(warp - kBuildWarps), (uint32_t)lane, deadline, kmin, kmax};
      ok = epilogue<kTplM, kMethod, kPrec, kExt>(c);
      kmin = c.kmin;
      kmax = c.kmax;
      if (!ok) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    }
    gx += nx;
  }

  if constexpr (kTplM) {
    if (do_ext && warp >= kBuildWarps && warp < kMmaWarp && t_ok) {
      atomicMin(&p.ext[2 * (t0 + tl)], kmin);
      atomicMax(&p.ext[2 * (t0 + tl) + 1], kmax);
    }
  }
  __syncthreads();
  if (!kTplM && do_ext)
    for (uint32_t t = threadIdx.x; t < nt; t += kThreads) {
      atomicMin(&p.ext[2 * (t0 + t)], s_ext[2 * t]);
      atomicMax(&p.ext[2 * (t0 + t) + 1], s_ext[2 * t + 1]);
    }
  if (warp == kMmaWarp) {
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kWaitNs) && lane == 0) atomicMax(p.err, p.tag);
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

int sm_count() { return device_sm_count(); }

__global__ void many_keys_init_kernel(unsigned long long* keys, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    keys[2 * i] = ~0ull;
    keys[2 * i + 1] = 0ull;
  }
}

// keys of template t -> ipb_extremes_f32 (locations in the Wo-wide score map)
__global__ void many_keys_finish_kernel(const unsigned long long* keys, uint32_t Wo, ipb_extremes_f32* out,
                                        uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long kmin = keys[2 * i], kmax = keys[2 * i + 1];
  auto value = [](uint32_t ok) { return __uint_as_float((ok & 0x80000000u) ? (ok & 0x7FFFFFFFu) : ~ok); };
  const uint32_t imin = (uint32_t)kmin, imax = 0xFFFFFFFFu - (uint32_t)kmax;
  ipb_extremes_f32 r;
  r.max_value = value((uint32_t)(kmax >> 32));
  r.min_value = value((uint32_t)(kmin >> 32));
  r.max_value_location_x = imax % Wo;
  r.max_value_location_y = imax / Wo;
  r.min_value_location_x = imin % Wo;
  r.min_value_location_y = imin / Wo;
  out[i] = r;
}

// Shared-memory carve for a template block of nb; returns the total bytes.
uint32_t many_carve(ManyParams& p, uint32_t nb) {
  uint32_t off = 1024;
  p.b_off = off;
  off += (uint32_t)align_up((size_t)p.h * p.kw * nb, 128);
  p.tss_off = off;
  off += (uint32_t)align_up(4 * nb, 128);
  p.ext_off = off;
  off += (uint32_t)align_up(16 * nb, 128);
  p.img_off = off;
  off += (uint32_t)align_up((size_t)p.rows * p.ip, 128);
  p.strip_off = off;
  off += (uint32_t)align_up((size_t)kStrips * (p.kw / 16) * p.rows * 16, 128);
  p.y_off = off;
  off += kXT * kM * 4;
  p.v_off = off;
  off += (uint32_t)align_up((size_t)p.rows * kXT * 4, 128);
  p.ry_off = off;
  off += kEpiWarps * kPosW * 8;
  return off;
}

constexpr uint32_t kSmemLimit = 227u * 1024u;

using ManyKernel = void (*)(ManyParams);

template <bool kTplM, int kMethod>
ManyKernel many_kernel_m(bool fp64, bool ext) {
  if (!method_is_norm(kMethod) || fp64)
    return ext ? many_match_kernel<kTplM, kMethod, IPB_PRECISION_EXACT_FP64, true>
               : many_match_kernel<kTplM, kMethod, IPB_PRECISION_EXACT_FP64, false>;
  return ext ? many_match_kernel<kTplM, kMethod, IPB_PRECISION_EXACT_F32, true>
             : many_match_kernel<kTplM, kMethod, IPB_PRECISION_EXACT_F32, false>;
}

template <bool kTplM>
ManyKernel many_kernel_a(int method, bool fp64, bool ext) {
  switch (method) {
    case kSse:
      return many_kernel_m<kTplM, kSse>(fp64, ext);
    case kSseNorm:
      return many_kernel_m<kTplM, kSseNorm>(fp64, ext);
    case kCcorr:
      return many_kernel_m<kTplM, kCcorr>(fp64, ext);
    default:
      return many_kernel_m<kTplM, kCcorrNorm>(fp64, ext);
  }
}

ManyKernel many_kernel_for(bool tplm, int method, bool fp64, bool ext) {
  return tplm ? many_kernel_a<true>(method, fp64, ext) : many_kernel_a<false>(method, fp64, ext);
}

}  // namespace

cudaError_t launch_many_keys_init(unsigned long long* keys, uint32_t n, cudaStream_t s) {
  many_keys_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(keys, n);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

cudaError_t launch_many_keys_finish(const unsigned long long* keys, uint32_t Wo, ipb_extremes_f32* out, uint32_t n,
                                    cudaStream_t s) {
  many_keys_finish_kernel<<<(n + 255) / 256, 256, 0, s>>>(keys, Wo, out, n);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

bool many_supported(uint32_t w, uint32_t h, uint32_t n, int precision) {
  return precision != IPB_PRECISION_REFERENCE_F32 && w >= 16 && w <= 64 && h >= 1 && h <= 64 && n >= 1;
}

cudaError_t launch_many(const uint8_t* img, uint32_t W, uint32_t H, const uint8_t* tpl, uint32_t w, uint32_t h,
                        uint32_t n, int method, int precision, float* out, unsigned long long* ext_keys,
                        unsigned int* err, unsigned int tag, cudaStream_t stream, KernelTimer* timer) {
  ManyParams p{};
  p.img = img;
  p.W = W;
  p.H = H;
  p.tpl = tpl;
  p.w = w;
  p.h = h;
  p.n = n;
  p.kw = (w + 31) & ~31u;
  p.Wo = W - w + 1;
  p.Ho = H - h + 1;
  p.bands = (p.Ho + kM - 1) / kM;
  p.xtiles = (p.Wo + kXT - 1) / kXT;
  p.spatial = p.bands * p.xtiles;
  p.rows = kM + h - 1;
  p.ip = (uint32_t)align_up(kXT + p.kw + 16, 16);
  // templates as M when a block of 128 fits and the bank fills most of it;
  // otherwise the largest positions-as-M block (multiple of 16) that fits
  uint32_t smem = many_carve(p, 128);
  const bool tplm = smem <= kSmemLimit && n > 64;
  uint32_t nb = 128;
  if (!tplm) {
    for (nb = std::min(112u, (n + 15) & ~15u); nb >= 16; nb -= 16)
      if ((smem = many_carve(p, nb)) <= kSmemLimit) break;
    if (nb < 16) return cudaErrorNotSupported;
  }
  p.NB = nb;
  p.nblocks = (n + nb - 1) / nb;
  p.method = method;
  p.precision = precision;
  p.vec4 = ((n & 3u) == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) ? 1 : 0;
  p.img16 = ((reinterpret_cast<uintptr_t>(img) & 15u) == 0 && (W & 15u) == 0) ? 1 : 0;
  p.out = out;
  p.ext = ext_keys;
  p.err = err;
  p.tag = tag;
  p.wait_ns = pipeline_wait_ns();
  p.stall = pipeline_stall() ? 1u : 0u;
  static PerDeviceOnce attr;
  cudaError_t e = attr.run([] {
    cudaError_t r = cudaSuccess;
    for (int a = 0; a < 2 && r == cudaSuccess; ++a)
      for (int m = 0; m < 4 && r == cudaSuccess; ++m)
        for (int f = 0; f < 2 && r == cudaSuccess; ++f)
          for (int x = 0; x < 2 && r == cudaSuccess; ++x)
            r = cudaFuncSetAttribute(many_kernel_for(a != 0, m, f != 0, x != 0),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
    return r;
  });
  if (e != cudaSuccess) return e;
  // CTAs come in groups of nblocks (one per template block)
  uint32_t per = (uint32_t)sm_count() / p.nblocks;
  if (per < 1) per = 1;
  if (per > p.spatial) per = p.spatial;
  const uint32_t grid = per * p.nblocks;
  timer_begin(timer, kKernelMany, stream);
  many_kernel_for(tplm, method, precision == IPB_PRECISION_EXACT_FP64, ext_keys != nullptr)
      <<<grid, kThreads, smem, stream>>>(p);
  count_launch(kKernelMany);
  timer_end(timer, stream);
  return cudaGetLastError();
}

}  // namespace ipb
