// tm_learned.cu -- forward and backward kernels of the proposal network and
// its training step (layout and definition in tm_learned.cuh).
//
// The 32 -> 32 convolutions and the weight gradients run on bf16 tensor cores
// with fp32 accumulation (mma.sync m16n8k16, operands staged in shared memory
// and loaded with ldmatrix); layer 1 (one input channel, 9 taps), the
// embedding head of training, the softmax loss and Adam run on CUDA cores.
// Backward passes treat the bf16 roundings of the forward pass as the identity.
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

// ---- bf16 helpers ------------------------------------------------------------
__host__ __device__ __forceinline__ uint16_t f2bf(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7FFFu + ((u >> 16) & 1u);                                    // round to nearest even
  return (uint16_t)(u >> 16);
}
__host__ __device__ __forceinline__ float bf2f(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  return (uint32_t)f2bf(lo) | ((uint32_t)f2bf(hi) << 16);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
// D = A (16x16, row) * B (16x8, col) + D, bf16 in, fp32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---- weights -----------------------------------------------------------------
__global__ void pack_weights_kernel(const float* __restrict__ P, PackedWeights pw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // layers 2..5: 4 x 9 x 32 x 32 entries of each packed form
  if (i < 4 * 9 * kC * kC) {
    const int l = i / (9 * kC * kC), r = i % (9 * kC * kC);
    const int tap = r / (kC * kC), co = (r / kC) % kC, ci = r % kC;
    const float* W = P + w_off(l + 1);
    const int ky = tap / 3, kx = tap % 3;
    pw.fwd[i] = f2bf(W[((co * kC + ci) * 3 + ky) * 3 + kx]);
    // data gradient: out channel ci, in channel co, taps flipped
    pw.bwd[i] = f2bf(W[((ci * kC + co) * 3 + (2 - ky)) * 3 + (2 - kx)]);
  }
  if (i < kC * 9) pw.w1[i] = bf2f(f2bf(P[w_off(0) + i]));
  if (i < kLayers * kC) pw.bias[i] = P[b_off(i / kC) + i % kC];
}

// ---- layer 1 (downsample fused) ------------------------------------------------
constexpr int kT1 = 16;  // 16 x 16 downsampled pixels per block

// D tile (with a one-pixel halo) of image n at downsampled origin (ys0-1, xs0-1)
__device__ __forceinline__ void load_ds_tile(const uint8_t* __restrict__ img, uint32_t n, uint32_t h, uint32_t w,
                                             int ys0, int xs0, float (*s_d)[kT1 + 2]) {
  const int hs = (int)h / 4, ws = (int)w / 4;
  for (int i = threadIdx.x; i < (kT1 + 2) * (kT1 + 2); i += blockDim.x) {
    const int ty = i / (kT1 + 2), tx = i % (kT1 + 2);
    const int ys = ys0 - 1 + ty, xs = xs0 - 1 + tx;
    float v = 0.f;
    if (ys >= 0 && ys < hs && xs >= 0 && xs < ws) {
      const uint8_t* p = img + ((size_t)n * h + 4 * ys) * w + 4 * xs;
      int s = 0;
#pragma unroll
      for (int dy = 0; dy < 4; ++dy) {
        const uint32_t q = *reinterpret_cast<const uint32_t*>(p + (size_t)dy * w);
        s += (q & 0xFF) + ((q >> 8) & 0xFF) + ((q >> 16) & 0xFF) + (q >> 24);
      }
      v = (float)(s - 2048) * (1.0f / 1024.0f);
    }
    s_d[ty][tx] = v;
  }
}

__global__ void __launch_bounds__(256) conv1_kernel(const uint8_t* __restrict__ img, uint32_t h, uint32_t w,
                                                    const float* __restrict__ w1, const float* __restrict__ b1,
                                                    uint4* __restrict__ out) {
  __shared__ float s_d[kT1 + 2][kT1 + 2];
  __shared__ float s_w[kC * 9 + kC];
  const uint32_t n = blockIdx.z;
  const int ys0 = blockIdx.y * kT1, xs0 = blockIdx.x * kT1;
  for (int i = threadIdx.x; i < kC * 9; i += blockDim.x) s_w[i] = w1[i];
  if (threadIdx.x < kC) s_w[kC * 9 + threadIdx.x] = b1[threadIdx.x];
  load_ds_tile(img, n, h, w, ys0, xs0, s_d);
  __syncthreads();
  const int ty = threadIdx.x / kT1, tx = threadIdx.x % kT1;
  const int ys = ys0 + ty, xs = xs0 + tx;
  const uint32_t hs = h / 4, ws = w / 4;
  if (ys >= (int)hs || xs >= (int)ws) return;
  float d[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) d[k] = s_d[ty + k / 3][tx + k % 3];
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    uint32_t pk[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float v[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int co = 8 * c + 2 * j + e;
        float s = s_w[kC * 9 + co];
#pragma unroll
        for (int k = 0; k < 9; ++k) s = fmaf(s_w[co * 9 + k], d[k], s);
        v[e] = s > 0.f ? s : 0.f;
      }
      pk[j] = pack2(v[0], v[1]);
    }
    out[(((size_t)n * hs + ys) * kChunks + c) * ws + xs] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  }
}

// dW1[co][tap] += sum_p dZ1[p][co] D[p + tap - 1]; db1[co] += sum_p dZ1[p][co]
__global__ void __launch_bounds__(320) conv1_grad_kernel(const uint8_t* __restrict__ img, uint32_t h, uint32_t w,
                                                         const uint4* __restrict__ dz, float* __restrict__ dW1,
                                                         float* __restrict__ db1) {
  __shared__ float s_d[kT1 + 2][kT1 + 2];
  __shared__ float s_dz[kT1 * kT1][kC + 1];
  const uint32_t n = blockIdx.z;
  const int ys0 = blockIdx.y * kT1, xs0 = blockIdx.x * kT1;
  const uint32_t hs = h / 4, ws = w / 4;
  load_ds_tile(img, n, h, w, ys0, xs0, s_d);
  for (int i = threadIdx.x; i < kT1 * kT1 * kChunks; i += blockDim.x) {
    const int p = i / kChunks, c = i % kChunks;
    const int ys = ys0 + p / kT1, xs = xs0 + p % kT1;
    uint4 u = make_uint4(0u, 0u, 0u, 0u);
    if (ys < (int)hs && xs < (int)ws) u = dz[(((size_t)n * hs + ys) * kChunks + c) * ws + xs];
    const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      s_dz[p][8 * c + 2 * j] = bf2f((uint16_t)(wd[j] & 0xFFFF));
      s_dz[p][8 * c + 2 * j + 1] = bf2f((uint16_t)(wd[j] >> 16));
    }
  }
  __syncthreads();
  const int co = threadIdx.x / 10, which = threadIdx.x % 10;
  float acc = 0.f;
  for (int p = 0; p < kT1 * kT1; ++p) {
    const float g = s_dz[p][co];
    acc += which == 9 ? g : g * s_d[p / kT1 + which / 3][p % kT1 + which % 3];
  }
  if (acc != 0.f) {
    if (which == 9)
      atomicAdd(db1 + co, acc);
    else
      atomicAdd(dW1 + co * 9 + which, acc);
  }
}

// ---- 3x3 32 -> 32 convolution on tensor cores ----------------------------------
// Tile: 4 output rows x 64 pixels x 32 channels per block of 8 warps; warp w
// takes row w / 2, pixels 32 (w % 2) .. +32 as two 16-pixel m-tiles, all four
// 8-channel n-tiles. Per tap and 16-channel k step: A (pixels x channels) by
// ldmatrix from the staged input rows, B (channels x out channels) from the
// staged weights.
constexpr int kTH = 4, kTW = 64, kInW = kTW + 2, kWPitch = 40;  // weight rows: 32 bf16 + 8 pad (80 B)

struct ConvSmem {
  uint4 in[kTH + 2][kChunks][kInW];        // 25344 B; reused to stage the output
  uint16_t w[9][kC][kWPitch];               // 23040 B
};

__global__ void __launch_bounds__(256) conv_mma_kernel(const uint4* __restrict__ in, uint32_t H, uint32_t W,
                                                       const uint16_t* __restrict__ wt,
                                                       const float* __restrict__ bias, int relu,
                                                       const uint4* __restrict__ mask, uint4* __restrict__ out) {
  __shared__ __align__(16) ConvSmem sm;
  const uint32_t n = blockIdx.z;
  const int y0 = blockIdx.y * kTH, x0 = blockIdx.x * kTW;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < (kTH + 2) * kChunks * kInW; i += 256) {
    const int px = i % kInW, c = (i / kInW) % kChunks, r = i / (kInW * kChunks);
    const int y = y0 - 1 + r, x = x0 - 1 + px;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (y >= 0 && y < (int)H && x >= 0 && x < (int)W) v = in[(((size_t)n * H + y) * kChunks + c) * W + x];
    sm.in[r][c][px] = v;
  }
  for (int i = tid; i < 9 * kC * 4; i += 256) {
    const int q = i & 3, row = i >> 2;  // row = tap * 32 + co
    *reinterpret_cast<uint4*>(&sm.w[row / kC][row % kC][8 * q]) = reinterpret_cast<const uint4*>(wt)[i];
  }
  __syncthreads();

  const int wr = warp >> 1, wx = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;

  const int lrow = lane & 7, lm = lane >> 3;
#pragma unroll 1
  for (int tap = 0; tap < 9; ++tap) {
    const int ky = tap / 3, kx = tap % 3;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      uint32_t a[2][4];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int px = wx + 16 * m + kx + lrow + 8 * (lm & 1);
        ldsm_x4(smem_addr(&sm.in[wr + ky][2 * s + (lm >> 1)][px]), a[m][0], a[m][1], a[m][2], a[m][3]);
      }
      uint32_t b[4][2];
#pragma unroll
      for (int jp = 0; jp < 2; ++jp) {
        const int co = 8 * (2 * jp + (lm >> 1)) + lrow;
        ldsm_x4(smem_addr(&sm.w[tap][co][8 * (2 * s + (lm & 1))]), b[2 * jp][0], b[2 * jp][1], b[2 * jp + 1][0],
                b[2 * jp + 1][1]);
      }
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[m][j], a[m][0], a[m][1], a[m][2], a[m][3], b[j][0], b[j][1]);
    }
  }
  __syncthreads();  // the input tile is no longer read: stage the output in it
  uint32_t* stage = reinterpret_cast<uint32_t*>(&sm.in[0][0][0]);  // [kTH][4 chunks][kTW px][4 words]
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int co = 8 * j + 2 * t;
      const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
#pragma unroll
      for (int hlf = 0; hlf < 2; ++hlf) {
        float v0 = acc[m][j][2 * hlf] + b0, v1 = acc[m][j][2 * hlf + 1] + b1;
        if (relu) {
          v0 = v0 > 0.f ? v0 : 0.f;
          v1 = v1 > 0.f ? v1 : 0.f;
        }
        const int px = wx + 16 * m + g + 8 * hlf;
        stage[((wr * kChunks + j) * kTW + px) * 4 + t] = pack2(v0, v1);
      }
    }
  __syncthreads();
  for (int i = tid; i < kTH * kChunks * kTW; i += 256) {
    const int px = i % kTW, c = (i / kTW) % kChunks, r = i / (kTW * kChunks);
    const int y = y0 + r, x = x0 + px;
    if (y >= (int)H || x >= (int)W) continue;
    uint4 v = reinterpret_cast<const uint4*>(stage)[i];
    const size_t gi = (((size_t)n * H + y) * kChunks + c) * W + x;
    if (mask) {
      const uint4 mk = mask[gi];
      uint32_t* vw = reinterpret_cast<uint32_t*>(&v);
      const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bool lo = (int16_t)(mw[k] & 0xFFFF) > 0, hi = (int16_t)(mw[k] >> 16) > 0;
        vw[k] &= (lo ? 0x0000FFFFu : 0u) | (hi ? 0xFFFF0000u : 0u);
      }
    }
    out[gi] = v;
  }
}

// ---- weight gradients on tensor cores ----------------------------------------------
// dW[co][ci][ky][kx] += sum_p dZ[p][co] A[p + (ky-1, kx-1)][ci], db[co] += sum_p dZ[p][co]
// over a tile of 4 rows x 64 pixels: M = output channels (two m-tiles), N =
// input channels (four n-tiles), K = 16 pixels per step. The 18 (tap, m-tile)
// pairs are shared out over the 8 warps.
struct GradSmem {
  uint4 dz[kTH][kChunks][kTW];         // 16384 B
  uint4 a[kTH + 2][kChunks][kInW];     // 25344 B
};

__global__ void __launch_bounds__(256) conv_grad_kernel(const uint4* __restrict__ dz, const uint4* __restrict__ act,
                                                        uint32_t H, uint32_t W, float* __restrict__ dW,
                                                        float* __restrict__ db) {
  __shared__ __align__(16) GradSmem sm;
  const uint32_t n = blockIdx.z;
  const int y0 = blockIdx.y * kTH, x0 = blockIdx.x * kTW;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kTH * kChunks * kTW; i += 256) {
    const int px = i % kTW, c = (i / kTW) % kChunks, r = i / (kTW * kChunks);
    const int y = y0 + r, x = x0 + px;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (y < (int)H && x < (int)W) v = dz[(((size_t)n * H + y) * kChunks + c) * W + x];
    sm.dz[r][c][px] = v;
  }
  for (int i = tid; i < (kTH + 2) * kChunks * kInW; i += 256) {
    const int px = i % kInW, c = (i / kInW) % kChunks, r = i / (kInW * kChunks);
    const int y = y0 - 1 + r, x = x0 - 1 + px;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (y >= 0 && y < (int)H && x >= 0 && x < (int)W) v = act[(((size_t)n * H + y) * kChunks + c) * W + x];
    sm.a[r][c][px] = v;
  }
  __syncthreads();

  // bias gradient: thread (co, part) sums 32 of the tile's 256 pixels
  {
    const int co = tid & 31, part = tid >> 5;
    float s = 0.f;
    for (int p = part * 32; p < part * 32 + 32; ++p) {
      const uint4 u = sm.dz[p / kTW][co >> 3][p % kTW];
      const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
      const uint32_t word = wd[(co & 7) >> 1];
      s += bf2f((uint16_t)((co & 1) ? (word >> 16) : (word & 0xFFFF)));
    }
    if (s != 0.f) atomicAdd(db + co, s);
  }

  constexpr int kMaxPairs = 3;
  int npairs = 0;
  int ptap[kMaxPairs], pm[kMaxPairs];
#pragma unroll
  for (int k = 0; k < kMaxPairs; ++k) {
    const int q = warp + 8 * k;
    ptap[k] = q < 18 ? q >> 1 : 0;
    pm[k] = q & 1;
    if (q < 18) npairs = k + 1;
  }
  float acc[kMaxPairs][4][4];
#pragma unroll
  for (int k = 0; k < kMaxPairs; ++k)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[k][j][e] = 0.f;

  const int lrow = lane & 7, lm = lane >> 3;
#pragma unroll 1
  for (int r = 0; r < kTH; ++r) {
#pragma unroll 1
    for (int xs = 0; xs < kTW; xs += 16) {
      // A = dZ^T (out channels x pixels) of both m-tiles
      uint32_t a[2][4];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int px = xs + lrow + 8 * (lm >> 1);
        ldsm_x4_t(smem_addr(&sm.dz[r][2 * m + (lm & 1)][px]), a[m][0], a[m][1], a[m][2], a[m][3]);
      }
#pragma unroll
      for (int k = 0; k < kMaxPairs; ++k) {
        if (k >= npairs) break;
        const int ky = ptap[k] / 3, kx = ptap[k] % 3;
        uint32_t b[4][2];
#pragma unroll
        for (int jp = 0; jp < 2; ++jp) {
          const int px = xs + kx + lrow + 8 * (lm & 1);
          ldsm_x4_t(smem_addr(&sm.a[r + ky][2 * jp + (lm >> 1)][px]), b[2 * jp][0], b[2 * jp][1],
                    b[2 * jp + 1][0], b[2 * jp + 1][1]);
        }
        const uint32_t* am = a[pm[k]];
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[k][j], am[0], am[1], am[2], am[3], b[j][0], b[j][1]);
      }
    }
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k = 0; k < kMaxPairs; ++k) {
    if (k >= npairs) break;
    const int tap = ptap[k];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int co = 16 * pm[k] + g + 8 * (e >> 1), ci = 8 * j + 2 * t + (e & 1);
        if (acc[k][j][e] != 0.f) atomicAdd(dW + (co * kC + ci) * 9 + tap, acc[k][j][e]);
      }
  }
}

// ---- embedding, head and loss (training) ------------------------------------------------
__device__ __forceinline__ float act_at(const uint4* __restrict__ F, uint32_t n, uint32_t H, uint32_t W, int y, int x,
                                        int c) {
  if (y < 0 || y >= (int)H || x < 0 || x >= (int)W) return 0.f;
  const uint4 u = F[(((size_t)n * H + y) * kChunks + (c >> 3)) * W + x];
  const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
  const uint32_t word = wd[(c & 7) >> 1];
  return bf2f((uint16_t)((c & 1) ? (word >> 16) : (word & 0xFFFF)));
}

__global__ void embed_kernel(const uint4* __restrict__ Ft, uint32_t T, float* __restrict__ G) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T * kEmb) return;
  const uint32_t t = i / kEmb, o = (i % kEmb) / kC, c = i % kC;
  G[i] = act_at(Ft, t, kTplDs, kTplDs, kCentre + (int)(o >> 1), kCentre + (int)(o & 1), (int)c);
}

// z[t][p] = alpha sum_o F(p + o) . G[t][o] for the P = n * H * W positions of
// the crops (flat index ((k * H) + y) * W + x) and T <= 128 templates.
constexpr int kHeadPos = 32;
__global__ void __launch_bounds__(256) head_train_kernel(const uint4* __restrict__ F, uint32_t n, uint32_t H,
                                                         uint32_t W, const float* __restrict__ G, uint32_t T,
                                                         float* __restrict__ z) {
  extern __shared__ float sh[];
  float* s_f = sh;                          // [kHeadPos][kEmb + 1]
  float* s_g = sh + kHeadPos * (kEmb + 1);  // [T][kEmb]
  const size_t P = (size_t)n * H * W;
  const size_t p0 = (size_t)blockIdx.x * kHeadPos;
  for (int i = threadIdx.x; i < kHeadPos * kEmb; i += blockDim.x) {
    const int pi = i / kEmb, k = i % kEmb, o = k / kC, c = k % kC;
    const size_t p = p0 + pi;
    float v = 0.f;
    if (p < P) {
      const uint32_t x = (uint32_t)(p % W), y = (uint32_t)((p / W) % H), k2 = (uint32_t)(p / ((size_t)W * H));
      v = act_at(F, k2, H, W, (int)y + (o >> 1), (int)x + (o & 1), c);
    }
    s_f[pi * (kEmb + 1) + k] = v;
  }
  for (int i = threadIdx.x; i < (int)T * kEmb; i += blockDim.x) s_g[i] = G[i];
  __syncthreads();
  const int pi = threadIdx.x & 31;
  const size_t p = p0 + pi;
  for (uint32_t t = threadIdx.x >> 5; t < T; t += blockDim.x >> 5) {
    float s = 0.f;
    for (int k = 0; k < kEmb; ++k) s = fmaf(s_f[pi * (kEmb + 1) + k], s_g[t * kEmb + k], s);
    if (p < P) z[(size_t)t * P + p] = kAlpha * s;
  }
}

// per template (one block): with N_t the 3 x 3 neighbourhood of the positive
// pos_t inside its crop (a position one step from the target is as good a
// proposal, and the smooth scenes make neighbours nearly equal),
//   loss_t = logsumexp_{all p}(z_t) - logsumexp_{p in N_t}(z_t),
//   z_t <- dz_t = (softmax_all(z_t) - [p in N_t] softmax_{N_t}(z_t)) / T.
__device__ __forceinline__ bool in_nbhd(size_t p, size_t pt, uint32_t H, uint32_t W) {
  const size_t hw = (size_t)H * W;
  if (p / hw != pt / hw) return false;
  const int y = (int)((p % hw) / W), x = (int)(p % W), py = (int)((pt % hw) / W), px = (int)(pt % W);
  return y - py <= 1 && py - y <= 1 && x - px <= 1 && px - x <= 1;
}

__global__ void __launch_bounds__(1024) softmax_ce_kernel(float* __restrict__ z, size_t P, uint32_t H, uint32_t W,
                                                          const int64_t* __restrict__ pos, uint32_t T,
                                                          float* __restrict__ loss) {
  __shared__ float s_red[32];
  __shared__ float s_lsen;
  float* zt = z + (size_t)blockIdx.x * P;
  float mx = -INFINITY;
  for (size_t i = threadIdx.x; i < P; i += blockDim.x) mx = fmaxf(mx, zt[i]);
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : -INFINITY;
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) s_red[0] = v;
  }
  __syncthreads();
  mx = s_red[0];
  __syncthreads();
  float se = 0.f;
  for (size_t i = threadIdx.x; i < P; i += blockDim.x) se += expf(zt[i] - mx);
  for (int o = 16; o; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = se;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0.f;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) s_red[0] = v;
  }
  __syncthreads();
  const float lse = mx + logf(s_red[0]);
  const int64_t pt = pos[blockIdx.x];
  const bool pos_ok = pt >= 0 && (size_t)pt < P;  // an out-of-range positive makes the loss NaN
  if (threadIdx.x == 0) {
    float lsen = NAN;
    if (pos_ok) {
      const size_t hw = (size_t)H * W, base = (size_t)pt - (size_t)pt % hw;
      const int py = (int)(((size_t)pt % hw) / W), px = (int)((size_t)pt % W);
      float m = -INFINITY;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          if (py + dy >= 0 && py + dy < (int)H && px + dx >= 0 && px + dx < (int)W)
            m = fmaxf(m, zt[base + (size_t)(py + dy) * W + px + dx]);
      float e = 0.f;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          if (py + dy >= 0 && py + dy < (int)H && px + dx >= 0 && px + dx < (int)W)
            e += expf(zt[base + (size_t)(py + dy) * W + px + dx] - m);
      lsen = m + logf(e);
    }
    s_lsen = lsen;
  }
  __syncthreads();
  const float lsen = s_lsen;
  const float inv = 1.0f / (float)T;
  for (size_t i = threadIdx.x; i < P; i += blockDim.x) {
    const float zi = zt[i];
    float d = expf(zi - lse);
    if (pos_ok && in_nbhd(i, (size_t)pt, H, W)) d -= expf(zi - lsen);
    zt[i] = d * inv;
  }
  if (threadIdx.x == 0) atomicAdd(loss, (lse - lsen) * inv);
}

// dF[q][c] = alpha sum_o sum_t dz[t][q - o] G[t][o][c] (bf16, row-chunked)
__global__ void __launch_bounds__(256) head_grad_f_kernel(const float* __restrict__ dz, uint32_t n, uint32_t H,
                                                          uint32_t W, const float* __restrict__ G, uint32_t T,
                                                          uint4* __restrict__ dF) {
  extern __shared__ float sh[];
  float* s_g = sh;                 // [T][kEmb]
  float* s_dz = sh + T * kEmb;     // [4][kHeadPos][T]: dz at q - o
  const size_t P = (size_t)n * H * W;
  const size_t q0 = (size_t)blockIdx.x * kHeadPos;
  for (int i = threadIdx.x; i < (int)T * kEmb; i += blockDim.x) s_g[i] = G[i];
  for (int i = threadIdx.x; i < 4 * kHeadPos * (int)T; i += blockDim.x) {
    const int t = i % T, qi = (i / T) % kHeadPos, o = i / (T * kHeadPos);
    const size_t q = q0 + qi;
    float v = 0.f;
    if (q < P) {
      const int x = (int)(q % W) - (o & 1), y = (int)((q / W) % H) - (o >> 1);
      if (x >= 0 && y >= 0) v = dz[(size_t)t * P + (q - (o & 1) - (size_t)(o >> 1) * W)];
    }
    s_dz[i] = v;
  }
  __syncthreads();
  // thread (q, chunk): 8 channels
  const int qi = threadIdx.x >> 2, c8 = threadIdx.x & 3;
  if (qi >= kHeadPos) return;
  const size_t q = q0 + qi;
  if (q >= P) return;
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int o = 0; o < 4; ++o)
    for (uint32_t t = 0; t < T; ++t) {
      const float d = s_dz[(o * kHeadPos + qi) * T + t];
      if (d == 0.f) continue;
      const float* g = s_g + t * kEmb + o * kC + 8 * c8;
#pragma unroll
      for (int e = 0; e < 8; ++e) acc[e] = fmaf(d, g[e], acc[e]);
    }
  const uint32_t x = (uint32_t)(q % W), y = (uint32_t)((q / W) % H), k2 = (uint32_t)(q / ((size_t)W * H));
  dF[(((size_t)k2 * H + y) * kChunks + c8) * W + x] =
      make_uint4(pack2(kAlpha * acc[0], kAlpha * acc[1]), pack2(kAlpha * acc[2], kAlpha * acc[3]),
                 pack2(kAlpha * acc[4], kAlpha * acc[5]), pack2(kAlpha * acc[6], kAlpha * acc[7]));
}

// dG[t][k] += alpha sum_p dz[t][p] F4[p][k] over 256 positions per block
constexpr int kGradPos = 256, kGradSub = 32;
__global__ void __launch_bounds__(256) head_grad_g_kernel(const float* __restrict__ dz, const uint4* __restrict__ F,
                                                          uint32_t n, uint32_t H, uint32_t W, uint32_t T,
                                                          float* __restrict__ dG) {
  extern __shared__ float sh[];
  float* s_f = sh;                              // [kGradSub][kEmb]
  float* s_d = sh + kGradSub * kEmb;            // [T][kGradSub]
  const size_t P = (size_t)n * H * W;
  const size_t p0 = (size_t)blockIdx.x * kGradPos;
  // thread: output k = tid % 128, templates t = tid / 128, +2, ...
  const int k = threadIdx.x % kEmb, t0 = threadIdx.x / kEmb;
  float acc[64];
  const int nt = ((int)T - t0 + 1) / 2;
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.f;
  for (int sub = 0; sub < kGradPos; sub += kGradSub) {
    __syncthreads();
    for (int i = threadIdx.x; i < kGradSub * kEmb; i += blockDim.x) {
      const int pi = i / kEmb, kk = i % kEmb, o = kk / kC, c = kk % kC;
      const size_t p = p0 + sub + pi;
      float v = 0.f;
      if (p < P) {
        const uint32_t x = (uint32_t)(p % W), y = (uint32_t)((p / W) % H), k2 = (uint32_t)(p / ((size_t)W * H));
        v = act_at(F, k2, H, W, (int)y + (o >> 1), (int)x + (o & 1), c);
      }
      s_f[i] = v;
    }
    for (int i = threadIdx.x; i < (int)T * kGradSub; i += blockDim.x) {
      const int t = i / kGradSub, pi = i % kGradSub;
      const size_t p = p0 + sub + pi;
      s_d[i] = p < P ? dz[(size_t)t * P + p] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int pi = 0; pi < kGradSub; ++pi) {
      const float f = s_f[pi * kEmb + k];
#pragma unroll
      for (int i = 0; i < 64; ++i)
        if (i < nt) acc[i] = fmaf(s_d[(t0 + 2 * i) * kGradSub + pi], f, acc[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < 64; ++i)
    if (i < nt && acc[i] != 0.f) atomicAdd(dG + (size_t)(t0 + 2 * i) * kEmb + k, kAlpha * acc[i]);
}

// dFt (templates' 12 x 12 feature gradient, bf16 row-chunked): dG at the 2x2 centre, 0 elsewhere
__global__ void embed_grad_kernel(const float* __restrict__ dG, uint32_t T, uint4* __restrict__ dFt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;  // one 16-byte unit each
  if (i >= T * kTplDs * kChunks * kTplDs) return;
  const uint32_t x = i % kTplDs, c = (i / kTplDs) % kChunks, y = (i / (kTplDs * kChunks)) % kTplDs,
                 t = i / (kTplDs * kChunks * kTplDs);
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  const int oy = (int)y - kCentre, ox = (int)x - kCentre;
  if (oy >= 0 && oy < 2 && ox >= 0 && ox < 2) {
    const float* g = dG + (size_t)t * kEmb + (oy * 2 + ox) * kC + 8 * c;
    v = make_uint4(pack2(g[0], g[1]), pack2(g[2], g[3]), pack2(g[4], g[5]), pack2(g[6], g[7]));
  }
  dFt[i] = v;
}

// Adam on the fp32 parameter vector
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, uint32_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

cudaError_t launch_pack_weights(const float* params, PackedWeights pw, cudaStream_t s) {
  pack_weights_kernel<<<(4 * 9 * kC * kC + 255) / 256, 256, 0, s>>>(params, pw);
  count_launch(kKernelLearned);
  return cudaGetLastError();
}

cudaError_t launch_conv1(const uint8_t* img, uint32_t n, uint32_t h, uint32_t w, const float* w1, const float* b1,
                         uint4* out, cudaStream_t s) {
  const dim3 grid((w / 4 + kT1 - 1) / kT1, (h / 4 + kT1 - 1) / kT1, n);
  conv1_kernel<<<grid, kT1 * kT1, 0, s>>>(img, h, w, w1, b1, out);
  count_launch(kKernelLearned);
  return cudaGetLastError();
}

cudaError_t launch_conv_mma(const uint4* in, uint32_t n, uint32_t H, uint32_t W, const uint16_t* wt,
                            const float* bias, int relu, const uint4* mask, uint4* out, cudaStream_t s) {
  const dim3 grid((W + kTW - 1) / kTW, (H + kTH - 1) / kTH, n);
  conv_mma_kernel<<<grid, 256, 0, s>>>(in, H, W, wt, bias, relu, mask, out);
  count_launch(kKernelLearned);
  return cudaGetLastError();
}

cudaError_t launch_trunk(const uint8_t* img, uint32_t n, uint32_t h, uint32_t w, const PackedWeights& pw,
                         uint4* const* acts, uint4* tmp_a, uint4* tmp_b, uint4* F, cudaStream_t s, int kernel,
                         unsigned int* err, unsigned int tag) {
  const uint32_t H = h / 4, W = w / 4;
  uint4* cur = acts ? acts[0] : tmp_a;
  cudaError_t e = launch_conv1(img, n, h, w, pw.w1, pw.bias, cur, s);
  for (int l = 1; l < kLayers && e == cudaSuccess; ++l) {
    uint4* nxt = l == kLayers - 1 ? F : (acts ? acts[l] : (cur == tmp_a ? tmp_b : tmp_a));
    const uint16_t* wt = pw.fwd + (size_t)(l - 1) * 9 * kC * kC;
    const int relu = l < kLayers - 1 ? 1 : 0;
    e = kernel == 0 ? launch_conv_tc(cur, n, H, W, wt, pw.bias + l * kC, relu, nxt, err, tag, s)
                    : launch_conv_mma(cur, n, H, W, wt, pw.bias + l * kC, relu, nullptr, nxt, s);
    cur = nxt;
  }
  return e;
}

cudaError_t launch_embed(const uint4* Ft, uint32_t T, float* G, cudaStream_t s) {
  embed_kernel<<<(T * kEmb + 255) / 256, 256, 0, s>>>(Ft, T, G);
  count_launch(kKernelLearned);
  return cudaGetLastError();
}

}  // namespace learned
}  // namespace ipb

// ============================================================================
// C ABI: the network object and its training step
// ============================================================================
using namespace ipb;
using namespace ipb::learned;

struct ipb_proposal_net {
  int device = -1;
  float* params = nullptr;   // fp32 master copy (kParams)
  float* grads = nullptr;    // kParams
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  uint64_t steps = 0;
  PackedWeights pw{};
  void* pw_block = nullptr;
  // training scratch (grow-only)
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // error word of the tcgen05 convolutions of training steps (after the
  // parameters in the same allocation) and the tag of the last step
  unsigned int* err = nullptr;
  unsigned int tag = 0;
};

namespace ipb {
namespace learned {
const PackedWeights& net_weights(const ipb_proposal_net* net) { return net->pw; }

bool learned_use_mma() {
  static const bool v = [] {
    const char* e = std::getenv("IPB_LEARNED_KERNELS");
    return e && std::strcmp(e, "mma") == 0;
  }();
  return v;
}
}  // namespace learned
}  // namespace ipb

namespace {

constexpr size_t kPwBytes = 2 * 4 * 9 * kC * kC * sizeof(uint16_t) + kC * 9 * sizeof(float) + kLayers * kC * sizeof(float);

ipb_status net_fail(ipb_status st, const std::string& msg) {
  report_error(st, msg.c_str());
  return st;
}
ipb_status net_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IPB_OK;
  (void)cudaGetLastError();
  return net_fail(e == cudaErrorMemoryAllocation ? IPB_ERR_OUT_OF_MEMORY : IPB_ERR_CUDA,
                  std::string(what) + ": " + cudaGetErrorString(e));
}
#define NET_CUDA(call, what)                        \
  do {                                              \
    const ipb_status st_ = net_cuda((call), what);  \
    if (st_ != IPB_OK) return st_;                  \
  } while (0)

// carve of the training scratch for N crops of sh x sw and T templates
struct TrainCarve {
  uint4* acts_s[4];  // A1..A4 of the scenes
  uint4* Fs;
  uint4* acts_t[4];
  uint4* Ft;
  uint4* d_a;        // data-gradient ping-pong (scene-sized)
  uint4* d_b;
  uint4* dt_a;       // (template-sized)
  uint4* dt_b;
  float* G;          // T x 128
  float* dG;         // T x 128
  float* z;          // T x P
  float* loss;       // 1
  size_t bytes;
};

TrainCarve carve(uint8_t* base, uint32_t N, uint32_t sh, uint32_t sw, uint32_t T) {
  TrainCarve c{};
  size_t off = 0;
  auto take = [&](size_t b) {
    uint8_t* p = base ? base + off : nullptr;
    off += align_up(b, 256);
    return p;
  };
  const size_t us = act_units(N, sh / 4, sw / 4) * 16, ut = act_units(T, kTplDs, kTplDs) * 16;
  for (int i = 0; i < 4; ++i) c.acts_s[i] = reinterpret_cast<uint4*>(take(us));
  c.Fs = reinterpret_cast<uint4*>(take(us));
  for (int i = 0; i < 4; ++i) c.acts_t[i] = reinterpret_cast<uint4*>(take(ut));
  c.Ft = reinterpret_cast<uint4*>(take(ut));
  c.d_a = reinterpret_cast<uint4*>(take(us));
  c.d_b = reinterpret_cast<uint4*>(take(us));
  c.dt_a = reinterpret_cast<uint4*>(take(ut));
  c.dt_b = reinterpret_cast<uint4*>(take(ut));
  c.G = reinterpret_cast<float*>(take((size_t)T * kEmb * 4));
  c.dG = reinterpret_cast<float*>(take((size_t)T * kEmb * 4));
  c.z = reinterpret_cast<float*>(take((size_t)T * N * (sh / 4) * (sw / 4) * 4));
  c.loss = reinterpret_cast<float*>(take(4));
  c.bytes = off;
  return c;
}

// backward through the trunk of one side (scenes or templates): dz5 in d0
ipb_status trunk_backward(ipb_proposal_net* net, const uint8_t* img, uint32_t n, uint32_t h, uint32_t w,
                          uint4* const* acts, uint4* d0, uint4* d1, cudaStream_t s, bool tc) {
  const uint32_t H = h / 4, W = w / 4;
  uint4* dz = d0;
  uint4* other = d1;
  for (int l = kLayers - 1; l >= 1; --l) {
    // weight gradient of layer l+1 (index l): dz x A_l
    const dim3 grid((W + kTW - 1) / kTW, (H + kTH - 1) / kTH, n);
    conv_grad_kernel<<<grid, 256, 0, s>>>(dz, acts[l - 1], H, W, net->grads + w_off(l), net->grads + b_off(l));
    count_launch(kKernelLearned);
    NET_CUDA(cudaGetLastError(), "weight gradient");
    // data gradient into A_l, times relu'(Z_l) = [A_l > 0]
    const uint16_t* wb = net->pw.bwd + (size_t)(l - 1) * 9 * kC * kC;
    NET_CUDA(tc ? launch_conv_tc(dz, n, H, W, wb, nullptr, 0, other, net->err, net->tag, s, acts[l - 1])
                : launch_conv_mma(dz, n, H, W, wb, nullptr, 0, acts[l - 1], other, s),
             "data gradient");
    std::swap(dz, other);
  }
  const dim3 g1((W + kT1 - 1) / kT1, (H + kT1 - 1) / kT1, n);
  conv1_grad_kernel<<<g1, 320, 0, s>>>(img, h, w, dz, net->grads + w_off(0), net->grads + b_off(0));
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "layer-1 gradient");
  return IPB_OK;
}

// forward, loss and gradients (into net->grads, zeroed first) of one batch
ipb_status loss_and_grads(ipb_proposal_net* net, const uint8_t* scenes, uint32_t N, uint32_t sh, uint32_t sw,
                          const uint8_t* templates, uint32_t T, const int64_t* pos, cudaStream_t s, float* h_loss) {
  if (N == 0 || T == 0 || T > 128 || sh % 4 || sw % 4 || sh < 8 || sw < 8)
    return net_fail(IPB_ERR_INVALID_ARGUMENT,
                    "training batches take 1..128 templates of 48 x 48 and scene crops whose sides are multiples "
                    "of 4 (at least 8)");
  const TrainCarve need = carve(nullptr, N, sh, sw, T);
  if (net->scratch_bytes < need.bytes) {
    NET_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (net->scratch) cudaFree(net->scratch);
    net->scratch = nullptr;
    net->scratch_bytes = 0;
    NET_CUDA(cudaMalloc(&net->scratch, need.bytes), "cudaMalloc (training scratch)");
    net->scratch_bytes = need.bytes;
  }
  const TrainCarve c = carve(static_cast<uint8_t*>(net->scratch), N, sh, sw, T);
  const uint32_t H = sh / 4, W = sw / 4;
  const size_t P = (size_t)N * H * W;
  NET_CUDA(cudaMemsetAsync(net->grads, 0, sizeof(float) * kParams, s), "memset");
  NET_CUDA(cudaMemsetAsync(c.loss, 0, sizeof(float), s), "memset");
  NET_CUDA(cudaMemsetAsync(c.dG, 0, sizeof(float) * T * kEmb, s), "memset");
  NET_CUDA(launch_pack_weights(net->params, net->pw, s), "pack weights");
  // the 32-channel convolutions and their data gradients on tcgen05 (or
  // mma.sync with IPB_LEARNED_KERNELS=mma); the weight gradients on mma.sync
  const bool tc = !learned_use_mma();
  const int kernel = tc ? 0 : 1;
  net->tag += 1;
  NET_CUDA(launch_trunk(scenes, N, sh, sw, net->pw, c.acts_s, nullptr, nullptr, c.Fs, s, kernel, net->err, net->tag),
           "scene trunk");
  NET_CUDA(launch_trunk(templates, T, kTpl, kTpl, net->pw, c.acts_t, nullptr, nullptr, c.Ft, s, kernel, net->err,
                        net->tag),
           "template trunk");
  NET_CUDA(launch_embed(c.Ft, T, c.G, s), "embedding");
  const size_t head_smem = sizeof(float) * (kHeadPos * (kEmb + 1) + T * kEmb);
  const unsigned nblk = (unsigned)((P + kHeadPos - 1) / kHeadPos);
  static PerDeviceOnce attr;
  NET_CUDA(attr.run([] {
             cudaError_t e = cudaFuncSetAttribute(head_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  200 * 1024);
             if (e == cudaSuccess)
               e = cudaFuncSetAttribute(head_grad_f_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
             return e;
           }),
           "kernel attributes");
  head_train_kernel<<<nblk, 256, head_smem, s>>>(c.Fs, N, H, W, c.G, T, c.z);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "head");
  softmax_ce_kernel<<<T, 1024, 0, s>>>(c.z, P, H, W, pos, T, c.loss);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "loss");
  const size_t gf_smem = sizeof(float) * (T * kEmb + 4 * kHeadPos * T);
  head_grad_f_kernel<<<nblk, 4 * kHeadPos, gf_smem, s>>>(c.z, N, H, W, c.G, T, c.d_a);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "head gradient (features)");
  const size_t gg_smem = sizeof(float) * (kGradSub * kEmb + T * kGradSub);
  head_grad_g_kernel<<<(unsigned)((P + kGradPos - 1) / kGradPos), 256, gg_smem, s>>>(c.z, c.Fs, N, H, W, T, c.dG);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "head gradient (embedding)");
  const uint32_t tu = T * kTplDs * kChunks * kTplDs;
  embed_grad_kernel<<<(tu + 255) / 256, 256, 0, s>>>(c.dG, T, c.dt_a);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "embedding gradient");
  ipb_status st = trunk_backward(net, scenes, N, sh, sw, c.acts_s, c.d_a, c.d_b, s, tc);
  if (st != IPB_OK) return st;
  st = trunk_backward(net, templates, T, kTpl, kTpl, c.acts_t, c.dt_a, c.dt_b, s, tc);
  if (st != IPB_OK) return st;
  if (h_loss) {
    unsigned int failed = 0;
    NET_CUDA(cudaMemcpyAsync(h_loss, c.loss, sizeof(float), cudaMemcpyDeviceToHost, s), "copy loss");
    NET_CUDA(cudaMemcpyAsync(&failed, net->err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s), "copy error word");
    NET_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (failed >= net->tag && failed != 0)
      return net_fail(IPB_ERR_TIMEOUT, "a training convolution timed out waiting on its pipeline");
  }
  return IPB_OK;
}

}  // namespace

IPB_API ipb_status ipb_proposal_net_create(const float* params, ipb_proposal_net** out) {
  if (!params || !out) return net_fail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  int dev = 0;
  NET_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  int major = 0;
  NET_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "cudaDeviceGetAttribute");
  if (major != 10) return net_fail(IPB_ERR_NO_DEVICE, "imageproc_b200 needs an sm_100 (B200) device");
  auto* net = new ipb_proposal_net();
  net->device = dev;
  cudaError_t e = cudaMalloc(&net->params, sizeof(float) * kParams * 4 + 16);
  if (e == cudaSuccess) e = cudaMalloc(&net->pw_block, kPwBytes);
  if (e != cudaSuccess) {
    if (net->params) cudaFree(net->params);
    delete net;
    return net_cuda(e, "cudaMalloc (network)");
  }
  net->grads = net->params + kParams;
  net->adam_m = net->params + 2 * kParams;
  net->adam_v = net->params + 3 * kParams;
  net->err = reinterpret_cast<unsigned int*>(net->params + 4 * kParams);
  uint8_t* pb = static_cast<uint8_t*>(net->pw_block);
  net->pw.fwd = reinterpret_cast<uint16_t*>(pb);
  net->pw.bwd = net->pw.fwd + 4 * 9 * kC * kC;
  net->pw.w1 = reinterpret_cast<float*>(net->pw.bwd + 4 * 9 * kC * kC);
  net->pw.bias = net->pw.w1 + kC * 9;
  e = cudaMemcpy(net->params, params, sizeof(float) * kParams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(net->adam_m, 0, sizeof(float) * 2 * kParams + 16);
  if (e == cudaSuccess) e = launch_pack_weights(net->params, net->pw, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaFree(net->params);
    cudaFree(net->pw_block);
    delete net;
    return net_cuda(e, "network set-up");
  }
  *out = net;
  return IPB_OK;
}

IPB_API ipb_status ipb_proposal_net_destroy(ipb_proposal_net* net) {
  if (!net) return IPB_OK;
  cudaSetDevice(net->device);
  cudaDeviceSynchronize();
  cudaFree(net->params);
  cudaFree(net->pw_block);
  if (net->scratch) cudaFree(net->scratch);
  delete net;
  return IPB_OK;
}

IPB_API ipb_status ipb_proposal_net_get_params(const ipb_proposal_net* net, float* out) {
  if (!net || !out) return net_fail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  NET_CUDA(cudaMemcpy(out, net->params, sizeof(float) * kParams, cudaMemcpyDeviceToHost), "copy parameters");
  return IPB_OK;
}

IPB_API ipb_status ipb_proposal_net_gradients(ipb_proposal_net* net, const uint8_t* d_scenes, uint32_t n_scenes,
                                              uint32_t scene_height, uint32_t scene_width,
                                              const uint8_t* d_templates, uint32_t n_templates,
                                              const int64_t* d_positives, float* h_loss, float* h_grads,
                                              void* stream) {
  if (!net || !d_scenes || !d_templates || !d_positives)
    return net_fail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float loss = 0.f;
  ipb_status st = loss_and_grads(net, d_scenes, n_scenes, scene_height, scene_width, d_templates, n_templates,
                                 d_positives, s, &loss);
  if (st != IPB_OK) return st;
  if (h_loss) *h_loss = loss;
  if (h_grads) {
    NET_CUDA(cudaMemcpyAsync(h_grads, net->grads, sizeof(float) * kParams, cudaMemcpyDeviceToHost, s),
             "copy gradients");
    NET_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
  return IPB_OK;
}

IPB_API ipb_status ipb_proposal_net_train_step(ipb_proposal_net* net, const uint8_t* d_scenes, uint32_t n_scenes,
                                               uint32_t scene_height, uint32_t scene_width,
                                               const uint8_t* d_templates, uint32_t n_templates,
                                               const int64_t* d_positives, float learning_rate, float* h_loss,
                                               void* stream) {
  if (!net || !d_scenes || !d_templates || !d_positives)
    return net_fail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ipb_status st = loss_and_grads(net, d_scenes, n_scenes, scene_height, scene_width, d_templates, n_templates,
                                 d_positives, s, h_loss);
  if (st != IPB_OK) return st;
  net->steps += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - (float)std::pow((double)b1, (double)net->steps);
  const float c2 = 1.f - (float)std::pow((double)b2, (double)net->steps);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(net->params, net->grads, net->adam_m, net->adam_v, kParams,
                                                    learning_rate, b1, b2, 1e-8f, c1, c2);
  count_launch(kKernelLearned);
  NET_CUDA(cudaGetLastError(), "adam");
  NET_CUDA(launch_pack_weights(net->params, net->pw, s), "pack weights");
  return IPB_OK;
}

IPB_API ipb_status ipb_proposal_net_features(ipb_proposal_net* net, const uint8_t* d_image, uint32_t width,
                                             uint32_t height, int kernel, void* d_out, void* stream) {
  if (!net || !d_image || !d_out) return net_fail(IPB_ERR_INVALID_ARGUMENT, "null argument");
  if (width % 4 || height % 4 || width == 0 || height == 0)
    return net_fail(IPB_ERR_INVALID_ARGUMENT, "image sides must be non-zero multiples of 4");
  if (kernel != 0 && kernel != 1) return net_fail(IPB_ERR_INVALID_ARGUMENT, "kernel must be 0 or 1");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = 2 * align_up(act_units(1, height / 4, width / 4) * 16, 256);
  if (net->scratch_bytes < bytes) {
    NET_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (net->scratch) cudaFree(net->scratch);
    net->scratch = nullptr;
    net->scratch_bytes = 0;
    NET_CUDA(cudaMalloc(&net->scratch, bytes), "cudaMalloc (feature scratch)");
    net->scratch_bytes = bytes;
  }
  uint4* a = static_cast<uint4*>(net->scratch);
  uint4* b = a + bytes / 2 / 16;
  NET_CUDA(launch_trunk(d_image, 1, height, width, net->pw, nullptr, a, b, static_cast<uint4*>(d_out), s, kernel),
           "trunk");
  return IPB_OK;
}
