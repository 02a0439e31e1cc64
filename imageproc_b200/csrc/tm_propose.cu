// tm_propose.cu -- learned proposals, exact verification and certification
// for many 48 x 48 templates against one large image (SumOfSquaredErrors).
//
// The reference answers "where does this template match best" by scoring
// every window (match_template, src/template_matching.rs:78-92) and taking
// find_extremes (:479-511): the first minimum in row-major order. Here:
//   1. the proposal network (tm_learned.cuh) scores every downsampled
//      position for every template: the heatmap z_t(p), reduced on the fly
//      to the maximum of each 8 x 8 cell (head_cells_kernel, bf16 tensor
//      cores, fp32 accumulation);
//   2. per template, the top-k cells and a confidence margin: the softmax
//      probability of the best cell minus that of the best cell not next to
//      it (topk_kernel);
//   3. a window of 32 x 32 positions around each proposal is scored exactly
//      (integer sums, the many-templates kernel's f32 rounding) and the first
//      minimum kept (verify_kernel);
//   4. certification: for SumOfSquaredErrors every window p satisfies
//      SSE(p) >= sum_b (S_I,b(p) - S_T,b)^2 / 144 over the 16 blocks b of
//      12 x 12 pixels of the template (Cauchy-Schwarz on each block), with
//      S the block sums. Over a block of positions, S_I,b lies between the
//      minimum and maximum of the image's 12 x 12 box sums there, which gives
//      a lower bound for the whole block from two tables built once per
//      image. Blocks whose bound exceeds the verified minimum cannot hold the
//      answer; the others must lie inside a verified window, or are verified
//      too, one warp per 4 x 4 block (verify_blocks_kernel, up to 16384
//      blocks per template) -- otherwise the template falls back;
//   5. templates whose margin is below the threshold, or that could not be
//      certified, are answered exhaustively: up to 8 of them by one
//      single-template tensor-core launch (extremes only), more by the
//      many-templates kernel.
// A certified answer equals find_extremes' minimum of the exhaustive map
// exactly: every position outside the verified set has a larger score.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "imageproc_b200.h"
#include "tm_internal.h"
#include "tm_learned.cuh"

#define IPB_API extern "C" __attribute__((visibility("default")))

namespace ipb {
namespace learned {
namespace {

constexpr int kCell = 8;          // heatmap cell: 8 x 8 downsampled positions
constexpr int kMaxTopK = 16;
constexpr int kWin = 32;          // verification window: 32 x 32 positions
constexpr int kBlk = 12;          // certification block: 12 x 12 positions
constexpr int kMaxExtra = 16384;  // most extra 4 x 4 blocks a template may verify
constexpr int kVerifyCtas = 4 * 148;  // blocks of threads sharing all templates' extra blocks
constexpr uint32_t kFallbackPerTemplate = 8;  // fallbacks up to this many use the single-template kernel
constexpr int kPatch = kWin + kTpl - 1;        // 79 image rows / columns per window
constexpr int kPatchPitch = 96;                // 16-byte multiple >= kPatch + 4

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__host__ __device__ __forceinline__ uint16_t f2bf(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
// f32 bits -> unsigned key with the same order (no NaNs here)
__host__ __device__ __forceinline__ uint32_t okey(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float okey_value(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

// ---- 1. heatmap cells --------------------------------------------------------------
// Block: 8 downsampled rows (one cell row) x 64 positions x 32 templates; warp
// w takes row w, four 16-position m-tiles and four 8-template n-tiles; the
// "taps" are the four offsets o of the 2x2 embedding.
constexpr int kHW = 64, kHInW = kHW + 1, kGPitch = 40;
struct HeadSmem {
  uint4 in[kCell + 1][kChunks][kHInW];   // 37440 B
  uint16_t g[4][32][kGPitch];            // 10240 B
};

__global__ void __launch_bounds__(256) head_cells_kernel(const uint4* __restrict__ F, uint32_t H, uint32_t W,
                                                         const uint16_t* __restrict__ gb, uint32_t T,
                                                         unsigned long long* __restrict__ cells) {
  __shared__ __align__(16) HeadSmem sm;
  const int y0 = blockIdx.y * kCell, x0 = blockIdx.x * kHW;
  const uint32_t t0 = blockIdx.z * 32;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < (kCell + 1) * kChunks * kHInW; i += 256) {
    const int px = i % kHInW, c = (i / kHInW) % kChunks, r = i / (kHInW * kChunks);
    const int y = y0 + r, x = x0 + px;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (y < (int)H && x < (int)W) v = F[((size_t)y * kChunks + c) * W + x];
    sm.in[r][c][px] = v;
  }
  for (int i = tid; i < 4 * 32 * 4; i += 256) {  // 4 offsets x 32 templates x 4 chunks of 8 channels
    const int q = i & 3, row = i >> 2, o = row / 32, tl = row % 32;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (t0 + tl < T) v = reinterpret_cast<const uint4*>(gb)[((size_t)o * T + t0 + tl) * 4 + q];
    *reinterpret_cast<uint4*>(&sm.g[o][tl][8 * q]) = v;
  }
  __syncthreads();

  float acc[4][4][4];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;
  const int lrow = lane & 7, lm = lane >> 3;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const int oy = o >> 1, ox = o & 1;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      uint32_t b[4][2];
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        const int tl = 8 * (2 * jp + (lm >> 1)) + lrow;
        ldsm_x4(smem_addr(&sm.g[o][tl][8 * (2 * s + (lm & 1))]), b[2 * jp][0], b[2 * jp][1], b[2 * jp + 1][0],
                b[2 * jp + 1][1]);
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        uint32_t a0, a1, a2, a3;
        const int px = 16 * m + ox + lrow + 8 * (lm & 1);
        ldsm_x4(smem_addr(&sm.in[warp + oy][2 * s + (lm >> 1)][px]), a0, a1, a2, a3);
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[m][j], a0, a1, a2, a3, b[j][0], b[j][1]);
      }
    }
  }
  // cell maxima: (order key of the logit, complement of the position) so that
  // ties go to the smaller position; the staged input is dead, so the cell
  // table lives in its first 2 KB
  __syncthreads();
  unsigned long long (*cell)[32] = reinterpret_cast<unsigned long long (*)[32]>(&sm.in[0][0][0]);
  for (int i = tid; i < (kHW / kCell) * 32; i += 256) (&cell[0][0])[i] = 0ull;
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  const int y = y0 + warp;
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int x = x0 + 16 * m + g + 8 * (e >> 1);
        unsigned long long key = 0ull;
        if (y < (int)H && x < (int)W)
          key = ((unsigned long long)okey(kAlpha * acc[m][j][e]) << 32) |
                (0xFFFFFFFFu - (uint32_t)((uint32_t)y * W + (uint32_t)x));
#pragma unroll
        for (int d = 4; d < 32; d <<= 1) {
          const unsigned long long o2 = __shfl_xor_sync(0xffffffffu, key, d);
          key = o2 > key ? o2 : key;
        }
        if (g == 0) atomicMax(&cell[2 * m + (e >> 1)][8 * j + 2 * t + (e & 1)], key);
      }
  __syncthreads();
  const uint32_t Cx = (W + kCell - 1) / kCell, Cy = (H + kCell - 1) / kCell;
  for (int i = tid; i < (kHW / kCell) * 32; i += 256) {
    const int tl = i / (kHW / kCell), cl = i % (kHW / kCell);
    const uint32_t cx = blockIdx.x * (kHW / kCell) + cl, cy = blockIdx.y;
    if (t0 + tl < T && cx < Cx && cy < Cy) cells[((size_t)(t0 + tl) * Cy + cy) * Cx + cx] = cell[cl][tl];
  }
}

// G (fp32, [T][o * 32 + c]) -> bf16 [o][T][c] for the head's B operand
__global__ void pack_embedding_kernel(const float* __restrict__ G, uint32_t T, uint16_t* __restrict__ gb) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T * kEmb) return;
  const uint32_t t = i / kEmb, o = (i % kEmb) / kC, c = i % kC;
  gb[((size_t)o * T + t) * kC + c] = f2bf(G[i]);
}

// ---- 2. top-k cells and margin ----------------------------------------------------
struct TopK {
  uint32_t pos[kMaxTopK];  // downsampled positions (y * W + x) of the best cells
  float logit[kMaxTopK];
  float margin;
  uint32_t count;
};

__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* red) {
  for (int d = 16; d; d >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, d);
    v = o > v ? o : v;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0ull;
    for (int d = 16; d; d >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, d);
      v = o > v ? o : v;
    }
    if (threadIdx.x == 0) red[32] = v;
  }
  __syncthreads();
  return red[32];
}

__device__ __forceinline__ float block_sum(float v, float* red) {
  for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if (threadIdx.x == 0) red[32] = v;
  }
  __syncthreads();
  return red[32];
}

// One block (512 threads) per template. One pass over the cells: every
// thread keeps the 16 largest keys it sees, sorted, in registers; then k
// block-wide maxima over the threads' list heads merge them (the owner of
// each maximum shifts its list). Keys are distinct (they hold the position).
// A second pass gives the softmax over all cells.
__global__ void __launch_bounds__(512) topk_kernel(const unsigned long long* __restrict__ cells, uint32_t Cy,
                                                    uint32_t Cx, uint32_t W, uint32_t k, TopK* __restrict__ out) {
  __shared__ unsigned long long red[33];
  __shared__ float redf[33];
  __shared__ uint32_t sel_cell[kMaxTopK];
  const unsigned long long* ct = cells + (size_t)blockIdx.x * Cy * Cx;
  const uint32_t nc = Cy * Cx;
  unsigned long long top[kMaxTopK];
  uint32_t topi[kMaxTopK];
#pragma unroll
  for (int j = 0; j < kMaxTopK; ++j) {
    top[j] = 0ull;
    topi[j] = 0u;
  }
  for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
    unsigned long long v = ct[i];
    uint32_t vi = i;
    if (v <= top[kMaxTopK - 1]) continue;
    // insert: carry the new key down the sorted list
#pragma unroll
    for (int j = 0; j < kMaxTopK; ++j) {
      if (v > top[j]) {
        const unsigned long long t = top[j];
        const uint32_t ti = topi[j];
        top[j] = v;
        topi[j] = vi;
        v = t;
        vi = ti;
      }
    }
  }
  TopK r;
  r.count = 0;
  for (uint32_t round = 0; round < k; ++round) {
    const unsigned long long m = block_max_u64(top[0], red);
    if (m == 0ull) break;
    if (top[0] == m) {
      sel_cell[round] = topi[0];
#pragma unroll
      for (int j = 0; j + 1 < kMaxTopK; ++j) {
        top[j] = top[j + 1];
        topi[j] = topi[j + 1];
      }
      top[kMaxTopK - 1] = 0ull;
    }
    r.pos[round] = 0xFFFFFFFFu - (uint32_t)(m & 0xFFFFFFFFu);
    r.logit[round] = okey_value((uint32_t)(m >> 32));
    r.count = round + 1;
  }
  __syncthreads();
  // margin: softmax probability of the best cell minus that of the best cell
  // that is not one of its 8 neighbours
  float margin = 0.f;
  if (r.count > 0) {
    const float z1 = r.logit[0];
    const uint32_t c1 = sel_cell[0], cy1 = c1 / Cx, cx1 = c1 % Cx;
    float se = 0.f;
    unsigned long long far = 0ull;
    for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
      const unsigned long long v = ct[i];
      se += expf(okey_value((uint32_t)(v >> 32)) - z1);
      const uint32_t cy = i / Cx, cx = i % Cx;
      const bool near = (cy + 1 >= cy1 && cy <= cy1 + 1 && cx + 1 >= cx1 && cx <= cx1 + 1);
      if (!near && v > far) far = v;
    }
    const float S = block_sum(se, redf);
    const unsigned long long f2 = block_max_u64(far, red);
    const float p2 = f2 ? expf(okey_value((uint32_t)(f2 >> 32)) - z1) / S : 0.f;
    margin = 1.f / S - p2;
  }
  r.margin = margin;
  if (threadIdx.x == 0) out[blockIdx.x] = r;
  (void)W;
}

// ---- 3. exact verification of rectangles of positions ------------------------------------
struct Rect {
  uint32_t x0, y0, w, h;  // positions [x0, x0 + w) x [y0, y0 + h), w, h <= 32
};

// One block per (rectangle, template): the image patch and the template in
// shared memory; thread (row r, 4-position group) sums X = sum I*T with dp4a
// over aligned image words shifted by byte_perm, Y from row prefix sums of
// I^2, and SSE = Y - 2X + TSS in integers, rounded once to f32 (the
// many-templates kernel's EXACT_FP64 SumOfSquaredErrors). The first minimum
// (order key of the score, then the position index) goes to best[t].
__global__ void __launch_bounds__(256) verify_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t H,
                                                     const uint8_t* __restrict__ tpl, const Rect* __restrict__ rects,
                                                     const uint32_t* __restrict__ counts, uint32_t max_rects,
                                                     unsigned long long* __restrict__ best) {
  __shared__ __align__(16) uint8_t s_img[kPatch][kPatchPitch];
  __shared__ uint32_t s_tpl[kTpl][kTpl / 4];
  __shared__ uint32_t s_sq[kPatch][kPatch + 1];  // prefix sums of I^2 per row
  __shared__ unsigned long long s_best[8];
  __shared__ unsigned long long s_tss;
  const uint32_t t = blockIdx.y;
  if (blockIdx.x >= min(counts[t], max_rects)) return;
  const Rect rc = rects[(size_t)t * max_rects + blockIdx.x];
  const uint32_t Wo = W - kTpl + 1;
  const uint8_t* tp = tpl + (size_t)t * kTpl * kTpl;
  const uint32_t pw = rc.w + kTpl - 1, ph = rc.h + kTpl - 1;
  for (uint32_t i = threadIdx.x; i < ph * kPatchPitch; i += blockDim.x) {
    const uint32_t r = i / kPatchPitch, c = i % kPatchPitch;
    s_img[r][c] = (c < pw) ? img[(size_t)(rc.y0 + r) * W + rc.x0 + c] : 0;
  }
  for (uint32_t i = threadIdx.x; i < kTpl * kTpl / 4; i += blockDim.x)
    s_tpl[i / (kTpl / 4)][i % (kTpl / 4)] = reinterpret_cast<const uint32_t*>(tp)[i];
  if (threadIdx.x == 0) s_tss = 0ull;
  __syncthreads();
  {
    unsigned long long part = 0ull;
    for (uint32_t i = threadIdx.x; i < kTpl * kTpl; i += blockDim.x) {
      const uint32_t v = tp[i];
      part += v * v;
    }
    for (int d = 16; d; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_tss, part);
  }
  // row prefix sums of I^2 (one warp per row)
  for (uint32_t r = threadIdx.x >> 5; r < ph; r += blockDim.x >> 5) {
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < pw; c0 += 32) {
      const uint32_t c = c0 + (threadIdx.x & 31);
      const uint32_t v = c < pw ? (uint32_t)s_img[r][c] * s_img[r][c] : 0u;
      uint32_t incl = v;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if ((int)(threadIdx.x & 31) >= d) incl += o;
      }
      if (c < pw) s_sq[r][c + 1] = carry + incl;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if ((threadIdx.x & 31) == 0) s_sq[r][0] = 0;
  }
  __syncthreads();
  const unsigned long long tss = s_tss;
  unsigned long long mykey = ~0ull;
  // work items: (row r, group of 4 positions starting at 4 gq)
  const uint32_t groups = (rc.w + 3) / 4;
  for (uint32_t it = threadIdx.x; it < rc.h * groups; it += blockDim.x) {
    const uint32_t r = it / groups, x4 = 4 * (it % groups);
    uint32_t X[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
    for (uint32_t dy = 0; dy < (uint32_t)kTpl; ++dy) {
      const uint32_t* row = reinterpret_cast<const uint32_t*>(&s_img[r + dy][0]) + (x4 >> 2);
      const uint32_t* trow = &s_tpl[dy][0];
      uint32_t cur = row[0];
#pragma unroll
      for (int k2 = 0; k2 < kTpl / 4; ++k2) {
        const uint32_t nxt = row[k2 + 1];
        const uint32_t tw = trow[k2];
        X[0] = __dp4a(cur, tw, X[0]);
        X[1] = __dp4a(__byte_perm(cur, nxt, 0x4321), tw, X[1]);
        X[2] = __dp4a(__byte_perm(cur, nxt, 0x5432), tw, X[2]);
        X[3] = __dp4a(__byte_perm(cur, nxt, 0x6543), tw, X[3]);
        cur = nxt;
      }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint32_t xl = x4 + s;
      if (xl >= rc.w) break;
      unsigned long long Y = 0ull;
      for (uint32_t dy = 0; dy < (uint32_t)kTpl; ++dy) Y += s_sq[r + dy][xl + kTpl] - s_sq[r + dy][xl];
      const unsigned long long sse = Y + tss - 2ull * X[s];
      const float score = (float)sse;  // round to nearest
      const uint32_t idx = (rc.y0 + r) * Wo + rc.x0 + xl;
      const unsigned long long key = ((unsigned long long)okey(score) << 32) | idx;
      mykey = key < mykey ? key : mykey;
    }
  }
  for (int d = 16; d; d >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, mykey, d);
    mykey = o < mykey ? o : mykey;
  }
  if ((threadIdx.x & 31) == 0) s_best[threadIdx.x >> 5] = mykey;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long b = s_best[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) b = s_best[i] < b ? s_best[i] : b;
    atomicMin(best + t, b);
  }
  (void)H;
}

// rectangles of the top-k windows: 32 x 32 positions centred on each
// proposal's full-resolution estimate 4 (p - 5) + 2, moved inside the map
__global__ void windows_kernel(const TopK* __restrict__ tk, uint32_t T, uint32_t Ws, uint32_t Wo, uint32_t Ho,
                               Rect* __restrict__ rects, uint32_t* __restrict__ counts, uint32_t max_rects,
                               unsigned long long* __restrict__ best, uint32_t* __restrict__ n_extra) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const TopK& r = tk[t];
  const uint32_t ww = Wo < (uint32_t)kWin ? Wo : kWin, wh = Ho < (uint32_t)kWin ? Ho : kWin;
  for (uint32_t i = 0; i < r.count; ++i) {
    const int px = (int)(r.pos[i] % Ws), py = (int)(r.pos[i] / Ws);
    int cx = 4 * (px - kCentre) + 2 - kWin / 2, cy = 4 * (py - kCentre) + 2 - kWin / 2;
    cx = cx < 0 ? 0 : (cx > (int)(Wo - ww) ? (int)(Wo - ww) : cx);
    cy = cy < 0 ? 0 : (cy > (int)(Ho - wh) ? (int)(Ho - wh) : cy);
    rects[(size_t)t * max_rects + i] = Rect{(uint32_t)cx, (uint32_t)cy, ww, wh};
  }
  counts[t] = r.count;
  best[t] = ~0ull;
  n_extra[t] = 0;
}

// ---- 4. certification tables ----------------------------------------------------------
// B(q) = the 12 x 12 box sum of the image at origin q (q.x <= W - 12, q.y <=
// H - 12). The micro table holds, for every 4 x 4 block of origins (micro
// block m = q / 4), the minimum and maximum of B over the block, packed as
// min | max << 16 (B <= 36720 fits 16 bits). For a block of positions P
// (4 x 4 positions at 4 P) and the template's 12 x 12 block b = (i, j), the
// origins p + 12 b lie in micro block P + 3 b -- aligned, since 12 = 3 x 4.
// Two coarser tables give the minimum and maximum over 4 x 4 micro blocks
// (16 x 16 positions) and over 16 x 16 micro blocks (64 x 64 positions)
// starting at each micro block.
constexpr int kTile = 64;  // origins per table tile side (16 x 16 micro blocks)

__global__ void __launch_bounds__(256) micro_table_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t H,
                                                          uint32_t Mx, uint32_t My, uint32_t* __restrict__ micro) {
  constexpr uint32_t kIn = kTile + kBlk - 1;  // 75 image rows and columns per tile
  constexpr uint32_t kRun = 16;               // box sums per thread along a row or a column
  __shared__ uint8_t s_img[kIn][kIn + 1];
  __shared__ uint16_t s_row[kIn][kTile];      // 12-pixel row sums at each origin column
  const uint32_t qx0 = blockIdx.x * kTile, qy0 = blockIdx.y * kTile;
  const uint32_t Qx = W - kBlk + 1, Qy = H - kBlk + 1;  // box-sum origins
  for (uint32_t i = threadIdx.x; i < kIn * kIn; i += blockDim.x) {
    const uint32_t r = i / kIn, c = i % kIn, y = qy0 + r, x = qx0 + c;
    s_img[r][c] = (y < H && x < W) ? img[(size_t)y * W + x] : 0;
  }
  __syncthreads();
  // row sums: each thread slides a 12-pixel window over a run of 16 columns
  for (uint32_t i = threadIdx.x; i < kIn * (kTile / kRun); i += blockDim.x) {
    const uint32_t r = i / (kTile / kRun), c0 = (i % (kTile / kRun)) * kRun;
    uint32_t v = 0;
#pragma unroll
    for (int d = 0; d < kBlk; ++d) v += s_img[r][c0 + d];
    s_row[r][c0] = (uint16_t)v;
#pragma unroll
    for (uint32_t j = 1; j < kRun; ++j) {
      v += (uint32_t)s_img[r][c0 + j + kBlk - 1] - (uint32_t)s_img[r][c0 + j - 1];
      s_row[r][c0 + j] = (uint16_t)v;
    }
  }
  __syncthreads();
  // box sums: thread (column c, rows 16 g .. 16 g + 15) slides down its
  // column; each run covers four micro blocks, whose minimum and maximum
  // over their 4 columns are folded across 4 adjacent lanes
  const uint32_t c = threadIdx.x & (kTile - 1), g = threadIdx.x / kTile;
  const bool col_ok = qx0 + c < Qx;
  uint32_t v = 0;
#pragma unroll
  for (int d = 0; d < kBlk; ++d) v += s_row[kRun * g + d][c];
  uint32_t mn[4], mx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    mn[k] = 0xFFFFu;
    mx[k] = 0u;
  }
#pragma unroll
  for (uint32_t j = 0; j < kRun; ++j) {
    const uint32_t r = kRun * g + j;
    if (j > 0) v += (uint32_t)s_row[r + kBlk - 1][c] - (uint32_t)s_row[r - 1][c];
    if (col_ok && qy0 + r < Qy) {
      mn[j / 4] = min(mn[j / 4], v);
      mx[j / 4] = max(mx[j / 4], v);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  const uint32_t mxb = blockIdx.x * (kTile / 4) + c / 4;
  if ((c & 3u) == 0 && mxb < Mx) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t myb = blockIdx.y * (kTile / 4) + 4 * g + k;
      if (myb < My) micro[(size_t)myb * Mx + mxb] = mn[k] | (mx[k] << 16);
    }
  }
}

// out[m] = min / max of in over the 4 x 4 entries in[m + step * (a, b)],
// a, b = 0..3 (clipped at the edges)
__global__ void span_table_kernel(const uint32_t* __restrict__ in, uint32_t Mx, uint32_t My, uint32_t step,
                                  uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Mx * My) return;
  const uint32_t x = i % Mx, y = i / Mx;
  uint32_t mn = 0xFFFFu, mx = 0u;
  for (uint32_t b = 0; b < 4 && y + step * b < My; ++b)
    for (uint32_t a = 0; a < 4 && x + step * a < Mx; ++a) {
      const uint32_t v = in[(size_t)(y + step * b) * Mx + x + step * a];
      mn = min(mn, v & 0xFFFFu);
      mx = max(mx, v >> 16);
    }
  out[i] = mn | (mx << 16);
}

// ---- 4b. certification of one template -------------------------------------------------
__device__ __forceinline__ unsigned long long lb_term(uint32_t st, uint32_t packed) {
  const uint32_t lo = packed & 0xFFFFu, hi = packed >> 16;
  const uint32_t d = st < lo ? lo - st : (st > hi ? st - hi : 0u);
  return (unsigned long long)d * d;
}

constexpr int kCertSlices = 16;  // blocks of threads per template
constexpr uint32_t kMaxLevel2 = 65536;  // most 16 x 16 blocks a template may carry to the last level

// What the three certification levels share: the template's 16 block sums,
// the verified minimum, and the lower bound of a block of positions starting
// at micro block (px, py), template block b at micro offset 3 b, from a table.
struct CertCtx {
  uint32_t st[16];
  float sstar;
  bool skip;  // low margin: the template falls back without a certificate
};

__device__ __forceinline__ void cert_setup(CertCtx& cc, uint32_t* s_st, const uint8_t* tpl, const TopK& tk,
                                           float min_margin, unsigned long long best) {
  if (threadIdx.x < 16) {
    const uint8_t* tp = tpl;
    const uint32_t by = threadIdx.x >> 2, bx = threadIdx.x & 3;
    uint32_t s = 0;
    for (int dy = 0; dy < kBlk; ++dy)
      for (int dx = 0; dx < kBlk; ++dx) s += tp[(by * kBlk + dy) * kTpl + bx * kBlk + dx];
    s_st[threadIdx.x] = s;
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < 16; ++b) cc.st[b] = s_st[b];
  cc.sstar = okey_value((uint32_t)(best >> 32));
  cc.skip = tk.margin < min_margin || tk.count == 0;
}

__device__ __forceinline__ bool cert_excluded(const CertCtx& cc, const uint32_t* __restrict__ table, uint32_t Mx,
                                              uint32_t My, uint32_t px, uint32_t py) {
  unsigned long long num = 0ull;
#pragma unroll
  for (int b = 0; b < 16; ++b) {
    const uint32_t mx = px + 3 * (b & 3), my = py + 3 * (b >> 2);
    if (mx < Mx && my < My) num += lb_term(cc.st[b], __ldg(table + (size_t)my * Mx + mx));
  }
  // SSE is an integer >= num / 144; excluded when RN_f32(ceil(LB)) exceeds the minimum
  return (float)((num + 143ull) / 144ull) > cc.sstar;
}

// Level 1, grid (template, slice): every block of 64 x 64 positions (16 x 16
// micro blocks) whose bound does not exclude it goes to list1.
__global__ void __launch_bounds__(256) certify_l1_kernel(const uint8_t* __restrict__ tpl,
                                                         const TopK* __restrict__ tk, float min_margin,
                                                         const unsigned long long* __restrict__ best,
                                                         const uint32_t* __restrict__ span16, uint32_t Mx,
                                                         uint32_t My, uint32_t Pmx, uint32_t Pmy,
                                                         uint32_t* __restrict__ list1, uint32_t cap1,
                                                         uint32_t* __restrict__ n1) {
  __shared__ uint32_t s_st[16];
  const uint32_t t = blockIdx.x;
  CertCtx cc;
  cert_setup(cc, s_st, tpl + (size_t)t * kTpl * kTpl, tk[t], min_margin, best[t]);
  if (cc.skip) return;
  const uint32_t C3x = (Pmx + 15) / 16, C3y = (Pmy + 15) / 16;
  for (uint32_t q = blockIdx.y * blockDim.x + threadIdx.x; q < C3x * C3y; q += gridDim.y * blockDim.x) {
    const uint32_t px = 16 * (q % C3x), py = 16 * (q / C3x);
    if (cert_excluded(cc, span16, Mx, My, px, py)) continue;
    const uint32_t slot = atomicAdd(n1 + t, 1u);
    if (slot < cap1) list1[(size_t)t * cap1 + slot] = q;  // cap1 = C3x * C3y: never exceeded
  }
}

// Level 2: the 16 blocks of 16 x 16 positions inside each list1 entry; the
// ones not excluded go to list2 (more than kMaxLevel2: the template falls
// back, recorded as an extra count above kMaxExtra).
__global__ void __launch_bounds__(256) certify_l2_kernel(const uint8_t* __restrict__ tpl,
                                                         const TopK* __restrict__ tk, float min_margin,
                                                         const unsigned long long* __restrict__ best,
                                                         const uint32_t* __restrict__ span4, uint32_t Mx,
                                                         uint32_t My, uint32_t Pmx, uint32_t Pmy,
                                                         const uint32_t* __restrict__ list1, uint32_t cap1,
                                                         const uint32_t* __restrict__ n1,
                                                         uint32_t* __restrict__ list2, uint32_t* __restrict__ n2,
                                                         uint32_t* __restrict__ n_extra) {
  __shared__ uint32_t s_st[16];
  const uint32_t t = blockIdx.x;
  CertCtx cc;
  cert_setup(cc, s_st, tpl + (size_t)t * kTpl * kTpl, tk[t], min_margin, best[t]);
  if (cc.skip) return;
  const uint32_t C3x = (Pmx + 15) / 16;
  const uint32_t work = min(n1[t], cap1) * 16u;
  for (uint32_t e = blockIdx.y * blockDim.x + threadIdx.x; e < work; e += gridDim.y * blockDim.x) {
    const uint32_t q = list1[(size_t)t * cap1 + (e >> 4)], k2 = e & 15u;
    const uint32_t px = 16 * (q % C3x) + 4 * (k2 & 3), py = 16 * (q / C3x) + 4 * (k2 >> 2);
    if (px >= Pmx || py >= Pmy || cert_excluded(cc, span4, Mx, My, px, py)) continue;
    const uint32_t slot = atomicAdd(n2 + t, 1u);
    if (slot < kMaxLevel2)
      list2[(size_t)t * kMaxLevel2 + slot] = py * Pmx + px;
    else
      atomicMax(n_extra + t, (uint32_t)kMaxExtra + 1u);
  }
}

// Level 3: the 16 micro blocks (4 x 4 positions) inside each list2 entry. A
// micro block that is neither excluded nor inside a verified window is
// appended to the template's extra list (counter n_extra[t]); a count above
// kMaxExtra means the template falls back.
__global__ void __launch_bounds__(256) certify_l3_kernel(const uint8_t* __restrict__ tpl,
                                                         const TopK* __restrict__ tk, float min_margin,
                                                         const unsigned long long* __restrict__ best,
                                                         const uint32_t* __restrict__ micro, uint32_t Mx,
                                                         uint32_t My, uint32_t Pmx, uint32_t Pmy, uint32_t Wo,
                                                         uint32_t Ho, const uint32_t* __restrict__ list2,
                                                         const uint32_t* __restrict__ n2,
                                                         const Rect* __restrict__ wins,
                                                         const uint32_t* __restrict__ nwin, uint32_t max_rects,
                                                         uint32_t* __restrict__ extra, uint32_t* __restrict__ n_extra) {
  __shared__ uint32_t s_st[16];
  __shared__ Rect s_win[kMaxTopK];
  const uint32_t t = blockIdx.x;
  const uint32_t nw = nwin[t];
  if (threadIdx.x < nw) s_win[threadIdx.x] = wins[(size_t)t * max_rects + threadIdx.x];
  CertCtx cc;
  cert_setup(cc, s_st, tpl + (size_t)t * kTpl * kTpl, tk[t], min_margin, best[t]);  // syncs s_win too
  if (cc.skip || n_extra[t] > (uint32_t)kMaxExtra) return;
  const uint32_t work = min(n2[t], kMaxLevel2) * 16u;
  for (uint32_t e = blockIdx.y * blockDim.x + threadIdx.x; e < work; e += gridDim.y * blockDim.x) {
    const uint32_t p2 = list2[(size_t)t * kMaxLevel2 + (e >> 4)], k1 = e & 15u;
    const uint32_t px = p2 % Pmx + (k1 & 3), py = p2 / Pmx + (k1 >> 2);
    if (px >= Pmx || py >= Pmy || cert_excluded(cc, micro, Mx, My, px, py)) continue;
    const uint32_t x0 = 4 * px, y0 = 4 * py;
    const uint32_t x1 = min(x0 + 4, Wo), y1 = min(y0 + 4, Ho);
    bool covered = false;
    for (uint32_t w = 0; w < nw && !covered; ++w) {
      const Rect r = s_win[w];
      covered = x0 >= r.x0 && y0 >= r.y0 && x1 <= r.x0 + r.w && y1 <= r.y0 + r.h;
    }
    if (covered) continue;
    const uint32_t slot = atomicAdd(n_extra + t, 1u);
    if (slot < kMaxExtra) extra[(size_t)t * kMaxExtra + slot] = py * Pmx + px;
  }
}

// offsets[t] = sum of the verified block counts of templates < t (a count
// above kMaxExtra counts 0: that template falls back), offsets[T] = total.
// One block of 1024 threads; templates in chunks of 1024.
__global__ void __launch_bounds__(1024) extra_offsets_kernel(const uint32_t* __restrict__ n_extra, uint32_t T,
                                                             uint32_t* __restrict__ offsets) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < T; base += blockDim.x) {
    const uint32_t t = base + threadIdx.x;
    uint32_t v = 0;
    if (t < T) {
      v = n_extra[t];
      v = v > (uint32_t)kMaxExtra ? 0u : v;
    }
    uint32_t incl = v;  // inclusive scan in the warp
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if ((int)lane >= d) incl += o;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
        if ((int)lane >= d) w += o;
      }
      s_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t before = s_carry + (warp ? s_warp[warp - 1] : 0u) + incl - v;
    if (t < T) offsets[t] = before;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) offsets[T] = s_carry;
}

// Exact minimum over the extra blocks of 4 x 4 positions (packed micro-block
// indices py * Pmx + px from certify_kernel) of every template whose list
// fits. All templates' blocks form one sequence (offsets from
// extra_offsets_kernel) that the grid's warps share in contiguous slices, so
// a template with many blocks is spread over the whole GPU. Per block, one
// warp stages the block's image patch (51 rows x 13 words; W is a multiple of
// 32 and 4 px a multiple of 4, so the words are aligned; words past the image
// read as zero and feed no valid position) in its own shared memory, then:
// R(r, ox) = sum of I^2 over 48 bytes of patch row r from column ox (51 x 4
// sums, dp4a), Y(ox, oy) = sum over 48 rows of R; X by lanes = 16 positions x
// 2 halves of the template's rows, dp4a on byte_perm-shifted patch words
// against the template staged in the warp's shared memory when the slice
// reaches a new template; the halves meet through one shuffle and SSE =
// Y - 2X + TSS rounds once to f32 as in verify_kernel. Each warp folds its
// first minimum per template into best[t].
constexpr int kPatchRows = 4 + kTpl - 1;        // 51
constexpr int kPatchWords = (4 + kTpl + 3) / 4;  // 13 (52 bytes >= 51)
constexpr int kVerifyWarps = 8;
__global__ void __launch_bounds__(kVerifyWarps * 32) verify_blocks_kernel(
    const uint8_t* __restrict__ img, uint32_t W, uint32_t H, const uint8_t* __restrict__ tpl,
    const uint32_t* __restrict__ extra, const uint32_t* __restrict__ offsets, uint32_t T, uint32_t Pmx,
    uint32_t Wo, uint32_t Ho, unsigned long long* __restrict__ best) {
  __shared__ uint32_t s_tpl[kVerifyWarps][kTpl][kTpl / 4 + 1];  // padded: the two row halves in different banks
  __shared__ uint32_t s_patch[kVerifyWarps][kPatchRows][kPatchWords];
  __shared__ uint32_t s_rsq[kVerifyWarps][kPatchRows][4];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t total = offsets[T];
  const uint32_t nwarps = gridDim.x * kVerifyWarps, gw = blockIdx.x * kVerifyWarps + warp;
  const uint32_t chunk = (total + nwarps - 1) / nwarps;
  const uint32_t beg = min(total, gw * chunk), end = min(total, beg + chunk);
  if (beg >= end) return;
  const uint32_t pos = lane & 15u, half = lane >> 4;
  const uint32_t ox = pos & 3u, oy = pos >> 2;
  const uint32_t sel = 0x3210u + ox * 0x1111u;
  const uint32_t* const img32 = reinterpret_cast<const uint32_t*>(img);
  const uint32_t wpr = W / 4;  // words per image row
  uint32_t (*tw)[kTpl / 4 + 1] = s_tpl[warp];
  uint32_t (*patch)[kPatchWords] = s_patch[warp];
  uint32_t (*rsq)[4] = s_rsq[warp];
  // the template of the slice's first block: offsets[t] <= beg < offsets[t + 1]
  uint32_t lo = 0, hi = T;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (offsets[mid] <= beg) lo = mid;
    else hi = mid;
  }
  uint32_t t = lo, t_end = offsets[t + 1];
  while (t_end <= beg) t_end = offsets[++t + 1];  // skip templates with no blocks
  bool staged = false;
  unsigned long long tss = 0ull, mykey = ~0ull;
  for (uint32_t i = beg; i < end; ++i) {
    if (i >= t_end || !staged) {
      if (staged) {  // the slice moves to the next template: fold this one's minimum
        for (int d = 16; d; d >>= 1) {
          const unsigned long long o = __shfl_xor_sync(0xffffffffu, mykey, d);
          mykey = o < mykey ? o : mykey;
        }
        if (lane == 0 && mykey != ~0ull) atomicMin(best + t, mykey);
        mykey = ~0ull;
        while (t_end <= i) t_end = offsets[++t + 1];
      }
      __syncwarp();  // the previous template's words are no longer read
      const uint32_t* src = reinterpret_cast<const uint32_t*>(tpl + (size_t)t * kTpl * kTpl);
      uint32_t part = 0;
      for (uint32_t e = lane; e < (uint32_t)(kTpl * kTpl / 4); e += 32) {
        const uint32_t v = __ldg(src + e);
        tw[e / (kTpl / 4)][e % (kTpl / 4)] = v;
        part = __dp4a(v, v, part);
      }
      for (int d = 16; d; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
      tss = part;  // at most 2304 * 65025 < 2^32
      staged = true;
    }
    const uint32_t mb = extra[(size_t)t * kMaxExtra + (i - offsets[t])];
    const uint32_t x0 = 4 * (mb % Pmx), y0 = 4 * (mb / Pmx);
    __syncwarp();  // the previous block's reads of the patch are done
    for (uint32_t e = lane; e < (uint32_t)(kPatchRows * kPatchWords); e += 32) {
      const uint32_t r = e / kPatchWords, c = e % kPatchWords;
      const uint32_t y = y0 + r, xw = x0 / 4 + c;
      patch[r][c] = (y < H && xw < wpr) ? __ldg(img32 + (size_t)y * wpr + xw) : 0u;
    }
    __syncwarp();
    // R(r, ox): squares of 48 bytes of row r from column ox
    for (uint32_t e = lane; e < (uint32_t)(kPatchRows * 4); e += 32) {
      const uint32_t r = e >> 2, o = e & 3u;
      const uint32_t sl = 0x3210u + o * 0x1111u;
      uint32_t acc = 0u, cur = patch[r][0];
#pragma unroll
      for (int k = 0; k < kTpl / 4; ++k) {
        const uint32_t nxt = patch[r][k + 1];
        const uint32_t iw = __byte_perm(cur, nxt, sl);
        acc = __dp4a(iw, iw, acc);
        cur = nxt;
      }
      rsq[r][o] = acc;
    }
    uint32_t X = 0u, Y = 0u;
#pragma unroll 2
    for (uint32_t dy = half * (kTpl / 2); dy < (half + 1) * (kTpl / 2); ++dy) {
      const uint32_t* prow = patch[oy + dy];
      uint32_t cur = prow[0];
#pragma unroll
      for (int k = 0; k < kTpl / 4; ++k) {
        const uint32_t nxt = prow[k + 1];
        X = __dp4a(__byte_perm(cur, nxt, sel), tw[dy][k], X);
        cur = nxt;
      }
    }
    __syncwarp();  // the square sums are written
#pragma unroll 4
    for (uint32_t dy = half * (kTpl / 2); dy < (half + 1) * (kTpl / 2); ++dy) Y += rsq[oy + dy][ox];
    X += __shfl_xor_sync(0xffffffffu, X, 16);
    Y += __shfl_xor_sync(0xffffffffu, Y, 16);
    const uint32_t x = x0 + ox, y = y0 + oy;
    if (x < Wo && y < Ho && half == 0) {
      const unsigned long long sse = (unsigned long long)Y + tss - 2ull * X;
      const float score = (float)sse;  // round to nearest
      const unsigned long long key = ((unsigned long long)okey(score) << 32) | (y * Wo + x);
      mykey = key < mykey ? key : mykey;
    }
  }
  for (int d = 16; d; d >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, mykey, d);
    mykey = o < mykey ? o : mykey;
  }
  if (lane == 0 && mykey != ~0ull) atomicMin(best + t, mykey);
}

// Windows of caller-given proposals: template origins (y * Wo + x, k per
// template), each the centre of a 32 x 32 window moved inside the map; the
// proposals carry no confidence (margin +inf: never below the threshold).
__global__ void origin_windows_kernel(const uint32_t* __restrict__ origins, uint32_t T, uint32_t k, uint32_t Wo,
                                      uint32_t Ho, TopK* __restrict__ tk, Rect* __restrict__ rects,
                                      uint32_t* __restrict__ counts, uint32_t max_rects,
                                      unsigned long long* __restrict__ best, uint32_t* __restrict__ n_extra) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const uint32_t ww = Wo < (uint32_t)kWin ? Wo : kWin, wh = Ho < (uint32_t)kWin ? Ho : kWin;
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t o = origins[(size_t)t * k + i];
    const uint32_t ox = o % Wo, oy = min(o / Wo, Ho - 1u);
    int cx = (int)ox - kWin / 2, cy = (int)oy - kWin / 2;
    cx = cx < 0 ? 0 : (cx > (int)(Wo - ww) ? (int)(Wo - ww) : cx);
    cy = cy < 0 ? 0 : (cy > (int)(Ho - wh) ? (int)(Ho - wh) : cy);
    rects[(size_t)t * max_rects + i] = Rect{(uint32_t)cx, (uint32_t)cy, ww, wh};
    tk[t].pos[i] = o;
    tk[t].logit[i] = 0.0f;
  }
  tk[t].margin = __int_as_float(0x7f800000);  // +inf
  tk[t].count = k;
  counts[t] = k;
  best[t] = ~0ull;
  n_extra[t] = 0;
}

}  // namespace
}  // namespace learned
}  // namespace ipb

// ============================================================================
// C ABI
// ============================================================================
using namespace ipb;
using namespace ipb::learned;

struct ipb_proposal_net;  // tm_learned.cu
namespace ipb {
namespace learned {
// network accessors (tm_learned.cu)
const PackedWeights& net_weights(const ipb_proposal_net* net);
}  // namespace learned
}  // namespace ipb

namespace {

ipb_status pfail(ipb_status st, const std::string& msg) {
  report_error(st, msg.c_str());
  return st;
}
ipb_status pcuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IPB_OK;
  (void)cudaGetLastError();
  return pfail(e == cudaErrorMemoryAllocation ? IPB_ERR_OUT_OF_MEMORY : IPB_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}
#define P_CUDA(call, what)                      \
  do {                                          \
    const ipb_status st_ = pcuda((call), what); \
    if (st_ != IPB_OK) return st_;              \
  } while (0)

struct ProposeScratch {
  int device = -1;
  void* p = nullptr;
  size_t bytes = 0;
  unsigned int* err = nullptr;
  unsigned int tag = 0;
  ~ProposeScratch() {
    if (device >= 0) {
      cudaSetDevice(device);
      cudaDeviceSynchronize();
      if (p) cudaFree(p);
      if (err) cudaFree(err);
    }
  }
};

struct Carve {
  uint4* a;
  uint4* b;
  uint4* F;
  uint4* ta;
  uint4* tb;
  uint4* Ft;
  float* G;
  uint16_t* gb;
  unsigned long long* cells;
  TopK* tk;
  Rect* wins;
  uint32_t* nwin;
  uint32_t* extra;  // per template: kMaxExtra packed micro-block indices
  uint32_t* n_extra;
  uint32_t* list1;  // certification work lists: per template cap1 64 x 64 blocks,
  uint32_t* list2;  // kMaxLevel2 16 x 16 blocks,
  uint32_t* n12;    // and their counts (n1: T words, then n2: T words)
  uint32_t* offsets;  // T + 1 prefix offsets of the verified extra blocks
  uint32_t cap1;
  unsigned long long* best;
  uint32_t* micro;
  uint32_t* span4;
  uint32_t* span16;
  uint8_t* fb_tpl;
  unsigned long long* fb_keys;
  ipb_extremes_f32* fb_ext;
  size_t bytes;
};

Carve carve(uint8_t* base, uint32_t W, uint32_t H, uint32_t T, uint32_t k) {
  Carve c{};
  size_t off = 0;
  auto take = [&](size_t b) {
    uint8_t* p = base ? base + off : nullptr;
    off += align_up(b ? b : 1, 256);
    return p;
  };
  const uint32_t Hs = H / 4, Ws = W / 4;
  const size_t su = act_units(1, Hs, Ws) * 16, tu = act_units(T, kTplDs, kTplDs) * 16;
  c.a = reinterpret_cast<uint4*>(take(su));
  c.b = reinterpret_cast<uint4*>(take(su));
  c.F = reinterpret_cast<uint4*>(take(su));
  c.ta = reinterpret_cast<uint4*>(take(tu));
  c.tb = reinterpret_cast<uint4*>(take(tu));
  c.Ft = reinterpret_cast<uint4*>(take(tu));
  c.G = reinterpret_cast<float*>(take((size_t)T * kEmb * 4));
  c.gb = reinterpret_cast<uint16_t*>(take((size_t)T * kEmb * 2));
  const uint32_t Cx = (Ws + kCell - 1) / kCell, Cy = (Hs + kCell - 1) / kCell;
  c.cells = reinterpret_cast<unsigned long long*>(take((size_t)T * Cx * Cy * 8));
  c.tk = reinterpret_cast<TopK*>(take((size_t)T * sizeof(TopK)));
  c.wins = reinterpret_cast<Rect*>(take((size_t)T * k * sizeof(Rect)));
  c.nwin = reinterpret_cast<uint32_t*>(take((size_t)T * 4));
  c.extra = reinterpret_cast<uint32_t*>(take((size_t)T * kMaxExtra * sizeof(uint32_t)));
  c.n_extra = reinterpret_cast<uint32_t*>(take((size_t)T * 4));
  {
    const uint32_t Pmx = (W - kTpl + 1 + 3) / 4, Pmy = (H - kTpl + 1 + 3) / 4;
    c.cap1 = ((Pmx + 15) / 16) * ((Pmy + 15) / 16);
  }
  c.list1 = reinterpret_cast<uint32_t*>(take((size_t)T * c.cap1 * 4));
  c.list2 = reinterpret_cast<uint32_t*>(take((size_t)T * kMaxLevel2 * 4));
  c.n12 = reinterpret_cast<uint32_t*>(take((size_t)T * 8));
  c.offsets = reinterpret_cast<uint32_t*>(take((size_t)(T + 1) * 4));
  c.best = reinterpret_cast<unsigned long long*>(take((size_t)T * 8));
  const uint32_t Mx = (W - kBlk + 1 + 3) / 4, My = (H - kBlk + 1 + 3) / 4;
  c.micro = reinterpret_cast<uint32_t*>(take((size_t)Mx * My * 4));
  c.span4 = reinterpret_cast<uint32_t*>(take((size_t)Mx * My * 4));
  c.span16 = reinterpret_cast<uint32_t*>(take((size_t)Mx * My * 4));
  c.fb_tpl = reinterpret_cast<uint8_t*>(take((size_t)T * kTpl * kTpl));
  c.fb_keys = reinterpret_cast<unsigned long long*>(take((size_t)T * 16));
  c.fb_ext = reinterpret_cast<ipb_extremes_f32*>(take((size_t)T * sizeof(ipb_extremes_f32)));
  c.bytes = off;
  return c;
}

bool use_mma_kernels() { return learned_use_mma(); }

ProposeScratch& scratch_for_thread() {
  thread_local ProposeScratch s;
  return s;
}


// Scratch of this thread for a query of W x H and T templates (grown, never shrunk).
ipb_status acquire_scratch(ProposeScratch& ps, size_t bytes) {
  int dev = 0;
  P_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (ps.device != dev || ps.bytes < bytes) {
    if (ps.p) {
      P_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
      cudaFree(ps.p);
      ps.p = nullptr;
      ps.bytes = 0;
    }
    if (ps.err && ps.device != dev) {
      cudaFree(ps.err);
      ps.err = nullptr;
    }
    ps.device = dev;
    P_CUDA(cudaMalloc(&ps.p, bytes), "cudaMalloc (proposal scratch)");
    ps.bytes = bytes;
    if (!ps.err) {
      P_CUDA(cudaMalloc(&ps.err, sizeof(unsigned int)), "cudaMalloc");
      P_CUDA(cudaMemset(ps.err, 0, sizeof(unsigned int)), "cudaMemset");
    }
  }
  return IPB_OK;
}

// Checks shared by the query entry points.
ipb_status check_query(const uint8_t* d_image, uint32_t W, uint32_t H, const uint8_t* d_templates,
                       uint32_t template_width, uint32_t template_height, int method, const char* who) {
  if (!d_image || !d_templates) return pfail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  if (template_width != (uint32_t)kTpl || template_height != (uint32_t)kTpl)
    return pfail(IPB_ERR_INVALID_ARGUMENT, std::string(who) + " take 48 x 48 templates");
  if (method != IPB_SUM_OF_SQUARED_ERRORS)
    return pfail(IPB_ERR_INVALID_ARGUMENT,
                 std::string(who) + " answer SumOfSquaredErrors queries (their certificate bounds that score)");
  if (W % 32 || H % 32 || W < 64 || H < 64)
    return pfail(IPB_ERR_INVALID_ARGUMENT, std::string(who) + " take images whose sides are multiples of 32 (>= 64)");
  if ((reinterpret_cast<uintptr_t>(d_image) | reinterpret_cast<uintptr_t>(d_templates)) & 15u)
    return pfail(IPB_ERR_INVALID_ARGUMENT, std::string(who) + " take 16-byte aligned image and template buffers");
  return IPB_OK;
}

// Steps 3 (after the windows are set) to 5: exact scores of the windows,
// certification, verdicts and the exhaustive fallback, into results.
ipb_status finish_queries(ProposeScratch& ps, const Carve& c, unsigned int call_tag, const uint8_t* d_image,
                          uint32_t W, uint32_t H, const uint8_t* d_templates, uint32_t T,
                          const ipb_propose_options& opt, ipb_proposal_result* results, cudaStream_t s) {
  const uint32_t Wo = W - kTpl + 1, Ho = H - kTpl + 1;
  const uint32_t Mx = (W - kBlk + 1 + 3) / 4, My = (H - kBlk + 1 + 3) / 4;
  verify_kernel<<<dim3(opt.top_k, T), 256, 0, s>>>(d_image, W, H, d_templates, c.wins, c.nwin, opt.top_k, c.best);
  count_launch(kKernelPropose);
  P_CUDA(cudaGetLastError(), "verification");
  // 4. certification
  if (opt.certify) {
    micro_table_kernel<<<dim3((Mx + 15) / 16, (My + 15) / 16), 256, 0, s>>>(d_image, W, H, Mx, My, c.micro);
    count_launch(kKernelPropose);
    span_table_kernel<<<(Mx * My + 255) / 256, 256, 0, s>>>(c.micro, Mx, My, 1, c.span4);
    count_launch(kKernelPropose);
    span_table_kernel<<<(Mx * My + 255) / 256, 256, 0, s>>>(c.span4, Mx, My, 4, c.span16);
    count_launch(kKernelPropose);
    const uint32_t Pmx = (Wo + 3) / 4, Pmy = (Ho + 3) / 4;
    P_CUDA(cudaMemsetAsync(c.n12, 0, (size_t)T * 8, s), "certification counters");
    certify_l1_kernel<<<dim3(T, kCertSlices), 256, 0, s>>>(d_templates, c.tk, opt.min_margin, c.best, c.span16, Mx, My,
                                                           Pmx, Pmy, c.list1, c.cap1, c.n12);
    count_launch(kKernelPropose);
    certify_l2_kernel<<<dim3(T, kCertSlices), 256, 0, s>>>(d_templates, c.tk, opt.min_margin, c.best, c.span4, Mx, My,
                                                           Pmx, Pmy, c.list1, c.cap1, c.n12, c.list2, c.n12 + T,
                                                           c.n_extra);
    count_launch(kKernelPropose);
    certify_l3_kernel<<<dim3(T, 4 * kCertSlices), 256, 0, s>>>(d_templates, c.tk, opt.min_margin, c.best, c.micro,
                                                               Mx, My, Pmx, Pmy, Wo, Ho, c.list2, c.n12 + T, c.wins,
                                                               c.nwin, opt.top_k, c.extra, c.n_extra);
    count_launch(kKernelPropose);
    extra_offsets_kernel<<<1, 1024, 0, s>>>(c.n_extra, T, c.offsets);
    count_launch(kKernelPropose);
    verify_blocks_kernel<<<kVerifyCtas, kVerifyWarps * 32, 0, s>>>(d_image, W, H, d_templates, c.extra, c.offsets, T,
                                                                   (Wo + 3) / 4, Wo, Ho, c.best);
    count_launch(kKernelPropose);
    P_CUDA(cudaGetLastError(), "certification");
  }
  // 5. the verdicts to the host; fallback templates through the exhaustive kernel
  std::vector<TopK> tk(T);
  std::vector<uint32_t> status(T, 0u), n_extra(T, 0u);
  std::vector<unsigned long long> best(T);
  P_CUDA(cudaMemcpyAsync(tk.data(), c.tk, sizeof(TopK) * T, cudaMemcpyDeviceToHost, s), "copy proposals");
  P_CUDA(cudaMemcpyAsync(best.data(), c.best, sizeof(unsigned long long) * T, cudaMemcpyDeviceToHost, s),
         "copy scores");
  if (opt.certify)
    P_CUDA(cudaMemcpyAsync(n_extra.data(), c.n_extra, sizeof(uint32_t) * T, cudaMemcpyDeviceToHost, s),
           "copy extra counts");
  unsigned int failed = 0;
  P_CUDA(cudaMemcpyAsync(&failed, ps.err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s), "copy error word");
  P_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  if (failed >= call_tag)
    return pfail(IPB_ERR_TIMEOUT, "a proposal-network convolution timed out waiting on its pipeline");
  std::vector<uint32_t> fb;
  for (uint32_t t = 0; t < T; ++t) {
    if (tk[t].margin < opt.min_margin || tk[t].count == 0)
      status[t] = 1;  // low margin: no verification counts
    else if (opt.certify && n_extra[t] > (uint32_t)kMaxExtra)
      status[t] = 2;  // too many blocks the bound cannot exclude
    if (status[t]) fb.push_back(t);
  }
  std::vector<ipb_extremes_f32> fb_ext(fb.size());
  if (!fb.empty()) {
    const uint32_t nf = (uint32_t)fb.size();
    P_CUDA(launch_many_keys_init(c.fb_keys, nf, s), "extremes init");
    if (nf <= kFallbackPerTemplate) {
      // a few templates: one single-template tensor-core launch over them
      // (its cost grows with the templates; the many-templates kernel's
      // hardly does below one block of templates)
      const uint8_t* tp[kFallbackPerTemplate];
      for (uint32_t i = 0; i < nf; ++i) tp[i] = d_templates + (size_t)fb[i] * kTpl * kTpl;
      P_CUDA(launch_umma_extremes(d_image, W, H, tp, nf, kTpl, kTpl, IPB_SUM_OF_SQUARED_ERRORS,
                                  IPB_PRECISION_EXACT_FP64, c.fb_keys, ps.err, call_tag, s),
             "exhaustive fallback");
    } else {
      for (size_t i = 0; i < fb.size(); ++i)
        P_CUDA(cudaMemcpyAsync(c.fb_tpl + i * kTpl * kTpl, d_templates + (size_t)fb[i] * kTpl * kTpl, kTpl * kTpl,
                               cudaMemcpyDeviceToDevice, s),
               "gather fallback templates");
      P_CUDA(launch_many(d_image, W, H, c.fb_tpl, kTpl, kTpl, nf, IPB_SUM_OF_SQUARED_ERRORS,
                         IPB_PRECISION_EXACT_FP64, nullptr, c.fb_keys, ps.err, call_tag, s, nullptr),
             "exhaustive fallback");
    }
    P_CUDA(launch_many_keys_finish(c.fb_keys, Wo, c.fb_ext, nf, s), "extremes finish");
    P_CUDA(cudaMemcpyAsync(fb_ext.data(), c.fb_ext, sizeof(ipb_extremes_f32) * nf, cudaMemcpyDeviceToHost, s),
           "copy fallback results");
    P_CUDA(cudaMemcpyAsync(&failed, ps.err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s), "copy error word");
    P_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (failed >= call_tag)
      return pfail(IPB_ERR_TIMEOUT, "the exhaustive fallback kernel timed out waiting on its pipeline");
  }
  size_t f = 0;
  for (uint32_t t = 0; t < T; ++t) {
    ipb_proposal_result& r = results[t];
    r.margin = tk[t].margin;
    r.path = status[t];
    r.uncertified = n_extra[t];
    if (status[t]) {
      const ipb_extremes_f32& e = fb_ext[f++];
      r.value = e.min_value;
      r.x = e.min_value_location_x;
      r.y = e.min_value_location_y;
    } else {
      const unsigned long long k = best[t];
      r.value = okey_value((uint32_t)(k >> 32));
      const uint32_t idx = (uint32_t)(k & 0xFFFFFFFFu);
      r.x = idx % Wo;
      r.y = idx / Wo;
    }
  }
  return IPB_OK;
}

}  // namespace

IPB_API ipb_status ipb_match_proposals_device(const uint8_t* d_image, uint32_t image_width, uint32_t image_height,
                                              const uint8_t* d_templates, uint32_t template_width,
                                              uint32_t template_height, uint32_t n_templates, int method,
                                              const uint32_t* d_origins, uint32_t k,
                                              const ipb_propose_options* options, ipb_proposal_result* results,
                                              void* stream) {
  const uint32_t W = image_width, H = image_height, T = n_templates;
  if (!results || (T && !d_origins)) return pfail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  ipb_status st = check_query(d_image, W, H, d_templates, template_width, template_height, method,
                              "proposal verification and certification");
  if (st != IPB_OK) return st;
  if (k == 0 || k > (uint32_t)kMaxTopK) return pfail(IPB_ERR_INVALID_ARGUMENT, "k must be 1..16");
  if (T == 0) return IPB_OK;
  ipb_propose_options opt{k, 0.1f, 1};
  if (options) opt = *options;
  opt.top_k = k;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ProposeScratch& ps = scratch_for_thread();
  if ((st = acquire_scratch(ps, carve(nullptr, W, H, T, k).bytes)) != IPB_OK) return st;
  const Carve c = carve(static_cast<uint8_t*>(ps.p), W, H, T, k);
  const unsigned int call_tag = ++ps.tag;
  origin_windows_kernel<<<(T + 127) / 128, 128, 0, s>>>(d_origins, T, k, W - kTpl + 1, H - kTpl + 1, c.tk, c.wins,
                                                        c.nwin, k, c.best, c.n_extra);
  count_launch(kKernelPropose);
  P_CUDA(cudaGetLastError(), "proposal windows");
  return finish_queries(ps, c, call_tag, d_image, W, H, d_templates, T, opt, results, s);
}

IPB_API ipb_status ipb_propose_and_match_device(const ipb_proposal_net* net, const uint8_t* d_image,
                                                uint32_t image_width, uint32_t image_height,
                                                const uint8_t* d_templates, uint32_t template_width,
                                                uint32_t template_height, uint32_t n_templates, int method,
                                                const ipb_propose_options* options, ipb_proposal_result* results,
                                                void* stream) {
  const uint32_t W = image_width, H = image_height, T = n_templates;
  if (!net || !results) return pfail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  {
    const ipb_status st = check_query(d_image, W, H, d_templates, template_width, template_height, method,
                                      "learned proposals");
    if (st != IPB_OK) return st;
  }
  if (T == 0) return IPB_OK;
  ipb_propose_options opt{16u, 0.1f, 1};
  if (options) opt = *options;
  if (opt.top_k == 0 || opt.top_k > (uint32_t)kMaxTopK)
    return pfail(IPB_ERR_INVALID_ARGUMENT, "top_k must be 1..16");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ProposeScratch& ps = scratch_for_thread();
  {
    const ipb_status st = acquire_scratch(ps, carve(nullptr, W, H, T, opt.top_k).bytes);
    if (st != IPB_OK) return st;
  }
  const Carve c = carve(static_cast<uint8_t*>(ps.p), W, H, T, opt.top_k);
  const PackedWeights& pw = net_weights(net);
  const uint32_t Hs = H / 4, Ws = W / 4, Wo = W - kTpl + 1, Ho = H - kTpl + 1;
  const uint32_t Cx = Ws / kCell, Cy = Hs / kCell;

  // 1. trunk of the image and of the templates, embedding, heatmap cells
  // one tag for every tensor-core launch of this call: a bounded wait that runs
  // out in any of them leaves a value >= it in the error word
  const unsigned int call_tag = ++ps.tag;
  const int conv_kernel = use_mma_kernels() ? 1 : 0;
  P_CUDA(launch_trunk(d_image, 1, H, W, pw, nullptr, c.a, c.b, c.F, s, conv_kernel, ps.err, call_tag),
         "image trunk");
  P_CUDA(launch_trunk(d_templates, T, kTpl, kTpl, pw, nullptr, c.ta, c.tb, c.Ft, s, conv_kernel, ps.err, call_tag),
         "template trunk");
  P_CUDA(launch_embed(c.Ft, T, c.G, s), "embedding");
  pack_embedding_kernel<<<(T * kEmb + 255) / 256, 256, 0, s>>>(c.G, T, c.gb);
  count_launch(kKernelPropose);
  if (use_mma_kernels()) {
    const dim3 hg((Ws + kHW - 1) / kHW, Hs / kCell, (T + 31) / 32);
    head_cells_kernel<<<hg, 256, 0, s>>>(c.F, Hs, Ws, c.gb, T, c.cells);
    count_launch(kKernelPropose);
    P_CUDA(cudaGetLastError(), "heatmap");
  } else {
    P_CUDA(launch_head_tc(c.F, Hs, Ws, c.gb, T, c.cells, ps.err, call_tag, s), "heatmap");
  }
  // 2. top-k and margins
  topk_kernel<<<T, 512, 0, s>>>(c.cells, Cy, Cx, Ws, opt.top_k, c.tk);
  count_launch(kKernelPropose);
  // 3. windows and their exact scores
  windows_kernel<<<(T + 127) / 128, 128, 0, s>>>(c.tk, T, Ws, Wo, Ho, c.wins, c.nwin, opt.top_k, c.best,
                                                 c.n_extra);
  count_launch(kKernelPropose);
  return finish_queries(ps, c, call_tag, d_image, W, H, d_templates, T, opt, results, s);
}
