// tm_many.cu -- many templates of one size against one image on tcgen05.
//
// The reference scores one template per call (match_template,
// src/template_matching.rs:78-92). For a bank of templates the work becomes
// one GEMM per output column x:
//   D[m][t] = sum_{dy,dx} I[y0 + m + dy][x + dx] * T_t[dy][dx]
// with M = 128 consecutive output rows, N = a block of NB templates and
// K = the template's pixels in (dy, dx) order, 32 bytes per MMA step.
//
// A operand: a "strip" of the image for column x -- for each 16-byte column
// chunk j, the rows y0 .. y0 + 127 + h - 1 of bytes [x + 16j, x + 16j + 16),
// stored 16 bytes per row in the canonical no-swizzle K-major layout. The A
// tile for template row dy is the same strip started dy rows (16*dy bytes)
// later, so one strip (about 5 KB) serves all h template rows.
// B operand: the template block, K-major, resident in shared memory for the
// CTA's lifetime. Every MMA is M128 x N128 x K32 (full tensor-core rate).
//
// Roles: 4 builder warps stage the image tile (cp.async), compute the window
// sums Y = sum I^2 of every position of the tile, and build strips; one warp
// issues the MMAs (elected lane); 8 epilogue warps read the accumulator
// (double-buffered in tensor memory), apply the method, write the scores and
// fold them into per-template extremes. Scores are position-major:
// out[(y * Wo + x) * n_templates + t], so each thread writes its 16
// consecutive template scores as one contiguous 64-byte run.
// Every wait is bounded (2 s) and reports through the error word.
#include "tm_common.cuh"
#include "tm_internal.h"
#include "tm_sm100.cuh"

namespace ipb {
namespace {

using namespace sm100;

constexpr int kM = 128;           // output rows per tile (tensor-memory lanes)
constexpr int kXT = 32;           // output columns per tile
constexpr int kBuildWarps = 4;
constexpr int kEpiWarps = 8;
constexpr int kMmaWarp = kBuildWarps + kEpiWarps;
constexpr int kThreads = (kMmaWarp + 1) * 32;
constexpr int kStrips = 3;
constexpr uint32_t kTmemCols = 256;  // two accumulators of up to 128 columns
constexpr unsigned long long kWaitNs = 2000000000ull;

struct ManyParams {
  const uint8_t* img;
  uint32_t W, H;
  const uint8_t* tpl;  // n templates of w x h, contiguous
  uint32_t w, h, n;
  uint32_t kw;       // w rounded up to 32
  uint32_t NB;       // templates per block (N of the MMA), multiple of 16, <= 128
  uint32_t nblocks;  // ceil(n / NB)
  uint32_t Wo, Ho, bands, xtiles, spatial;  // spatial tiles = bands * xtiles
  uint32_t rows;     // strip rows: 128 + h - 1
  uint32_t ip;       // staged image row pitch
  uint32_t b_off, tss_off, img_off, strip_off, y_off, v_off, ext_off;
  int method, precision, vec4;  // vec4: 16-byte score stores
  int img16;                    // image rows 16-byte aligned: cp.async staging
  float* out;                 // may be null (extremes only)
  unsigned long long* ext;    // 2 keys per template or null
  unsigned int* err;
  unsigned int tag;
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
      mbar_init(&sfull[s], kBuildWarps * 32);
      mbar_init(&sempty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      mbar_init(&dfull[d], 1);
      mbar_init(&dempty[d], kEpiWarps * 32);
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
  const uint32_t idesc = idesc_u8u8_s32(kM, p.NB);
  const bool do_ext = p.ext != nullptr;

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
    const unsigned long long deadline = global_ns() + kWaitNs;

    if (warp < kBuildWarps) {
      // strips: S_x[j][rho] = image row rho, bytes [xi + 16j, xi + 16j + 16)
      for (uint32_t xi = 0; xi < nx; ++xi) {
        const uint32_t g = gx + xi, s = g % kStrips;
        if (g >= kStrips && !mbar_wait_sleep(&sempty[s], ((g / kStrips) + 1) & 1u, deadline)) {
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
        mbar_arrive(&sfull[s]);
      }
      if (!ok) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    } else if (warp == kMmaWarp) {
      const bool leader = elect_one();
      const uint32_t lbo_a = p.rows * 16, lbo_b = p.NB * 16;
      for (uint32_t xi = 0; xi < nx; ++xi) {
        const uint32_t g = gx + xi, s = g % kStrips, d = g & 1u;
        const bool got_s = mbar_wait(&sfull[s], (g / kStrips) & 1u, deadline);
        const bool got_d = got_s && (g < 2 || mbar_wait(&dempty[d], ((g >> 1) + 1) & 1u, deadline));
        if (!__all_sync(0xffffffffu, got_s && got_d)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t a0 = smem_u32(s_strip + s * strip_bytes);
        const uint32_t b0 = smem_u32(bmat);
        if (leader) {
          uint32_t acc = 0;
          for (uint32_t dy = 0; dy < p.h; ++dy)
            for (uint32_t kk = 0; kk < p.kw / 32; ++kk) {
              const uint64_t ad = smem_desc_noswizzle(a0 + (2 * kk) * lbo_a + dy * 16, lbo_a, 128);
              const uint64_t bd = smem_desc_noswizzle(b0 + (dy * nch + 2 * kk) * lbo_b, lbo_b, 128);
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + d * 128),
                  "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                  : "memory");
              acc = 1u;
            }
          mma_commit(&sempty[s]);
          mma_commit(&dfull[d]);
        }
        __syncwarp();
      }
      if (!ok && lane == 0) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    } else {
      // epilogue warps: quadrant q of the lanes (output rows), half of the templates
      const uint32_t e = warp - kBuildWarps, q = e & 3, half = e >> 2;
      const uint32_t m = q * 32 + lane, y = y0 + m;
      const uint32_t ncol = p.NB / 2, c0 = half * ncol;
      for (uint32_t xi = 0; xi < nx; ++xi) {
        const uint32_t g = gx + xi, d = g & 1u;
        if (!mbar_wait_sleep(&dfull[d], (g >> 1) & 1u, deadline)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t x = x0 + xi;
        const uint32_t Y = s_y[xi * kM + m];
        const bool row_ok = y < p.Ho;
        float* orow = p.out ? p.out + ((size_t)y * p.Wo + x) * p.n + t0 : nullptr;
        for (uint32_t cc = c0; cc < c0 + ncol; cc += 16) {
          uint32_t v[16];
          tmem_ld16(tmem_addr(tmem, q * 32, d * 128 + cc), v);
          tmem_wait_ld();
          float f[16];
#pragma unroll
          for (int k = 0; k < 16; ++k) f[k] = finish_score32(p.method, p.precision, v[k], Y, s_tss[cc + k]);
          if (orow && row_ok) {
            if (p.vec4 && cc + 16 <= nt) {
#pragma unroll
              for (int k = 0; k < 16; k += 4)
                *reinterpret_cast<float4*>(orow + cc + k) = make_float4(f[k], f[k + 1], f[k + 2], f[k + 3]);
            } else {
              for (int k = 0; k < 16; ++k)
                if (cc + k < nt) orow[cc + k] = f[k];
            }
          }
          if (do_ext) {
            // per template: smallest / largest value over this warp's 32 rows,
            // the lowest row (= lowest linear index at this x) among ties
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              const uint32_t key = row_ok ? order_key(f[k]) : 0xFFFFFFFFu;
              const uint32_t kmn = __reduce_min_sync(0xffffffffu, key);
              const uint32_t ln = __ffs(__ballot_sync(0xffffffffu, key == kmn)) - 1;
              const uint32_t keyx = row_ok ? order_key(f[k]) : 0u;
              const uint32_t kmx = __reduce_max_sync(0xffffffffu, keyx);
              const uint32_t lx = __ffs(__ballot_sync(0xffffffffu, keyx == kmx)) - 1;
              if (lane == (uint32_t)k && cc + k < nt) {
                const uint32_t ymn = y0 + q * 32 + ln, ymx = y0 + q * 32 + lx;
                if (ymn < p.Ho) {
                  const unsigned long long kn = ((unsigned long long)kmn << 32) | (ymn * p.Wo + x);
                  atomicMin(&s_ext[2 * (cc + k)], kn);
                }
                if (ymx < p.Ho) {
                  const unsigned long long kx = ((unsigned long long)kmx << 32) | (0xFFFFFFFFu - (ymx * p.Wo + x));
                  atomicMax(&s_ext[2 * (cc + k) + 1], kx);
                }
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(&dempty[d]);
      }
      if (!ok) {
        *s_err = 1;
        atomicMax(p.err, p.tag);
      }
    }
    gx += nx;
  }

  __syncthreads();
  if (do_ext)
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
  // largest template block (multiple of 16, at most 128) whose carve fits
  uint32_t off = 0;
  uint32_t nb = 128;
  for (; nb >= 16; nb -= 16) {
    off = 1024;
    p.b_off = off;
    off += (uint32_t)align_up((size_t)h * p.kw * nb, 128);
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
    if (off <= 227u * 1024u) break;
  }
  if (nb < 16) return cudaErrorNotSupported;
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
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(many_match_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // CTAs come in groups of nblocks (one per template block)
  uint32_t per = (uint32_t)sm_count() / p.nblocks;
  if (per < 1) per = 1;
  if (per > p.spatial) per = p.spatial;
  const uint32_t grid = per * p.nblocks;
  timer_begin(timer, kKernelMany, stream);
  many_match_kernel<<<grid, kThreads, off, stream>>>(p);
  count_launch(kKernelMany);
  timer_end(timer, stream);
  return cudaGetLastError();
}

}  // namespace ipb
