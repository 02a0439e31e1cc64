// tm_exact_cc.cu -- exact-integer template matching on the CUDA cores.
//
// Computes, for every output position, the exact integer sums X = sum I*U and
// (masked) Y = sum I^2*V with dp4a (four u8 x u8 products per instruction),
// then applies the method's formula in the fused epilogue. Unmasked Y is the
// window sum of I^2 taken from the u64 integral image. Replaces the scalar
// f32 walk of methods::*::score_at (src/template_matching.rs:219-375) for
// small and medium templates; the tensor-core kernels take the large ones.
//
// Work decomposition: a block owns a 128 x TY tile of outputs (32 x 8
// threads, each thread 4 adjacent columns x RY rows). The template is walked
// in chunks of 16 rows x 64 columns; each chunk's template planes and the
// image rows it touches are staged in shared memory. Image words for the four
// column shifts come from one aligned word pair through byte_perm, and one
// image row feeds every (output row, template row) pair with equal sum, so
// each staged word is reused RY times.
//
// Per-chunk partial sums stay below 16*64*255*255 < 2^32 and are folded into
// u64 accumulators, so any template size is exact.
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

constexpr int kTX = 128;       // output columns per block
constexpr int kThreads = 256;  // 32 x 8
constexpr int kDYC = 16;       // template rows per chunk
constexpr int kDXC = 64;       // template columns per chunk
constexpr int kImgPitch = kTX + kDXC + 16;

// Plane sets. kVar 0: unmasked (I x T). 1: binary mask (I x Tm, L x m, H x m).
// 2: general mask (I x U0..U2, L x V0, L x V1, H x V0, H x V1).
template <int kVar> struct Planes;
template <> struct Planes<0> { static constexpr int NI = 1, NT = 1, NP = 1, RY = 4; };
template <> struct Planes<1> { static constexpr int NI = 3, NT = 2, NP = 3, RY = 2; };
template <> struct Planes<2> { static constexpr int NI = 3, NT = 5, NP = 7, RY = 1; };

// (image plane, template plane) of each product chain, per variant.
__device__ __forceinline__ void pair_planes(int var, int q, int& ip, int& tp) {
  if (var == 0) { ip = 0; tp = 0; return; }
  if (var == 1) {
    const int ips[3] = {0, 1, 2}, tps[3] = {0, 1, 1};
    ip = ips[q]; tp = tps[q]; return;
  }
  const int ips[7] = {0, 0, 0, 1, 1, 2, 2}, tps[7] = {0, 1, 2, 3, 4, 3, 4};
  ip = ips[q]; tp = tps[q];
}

template <int kVar>
__global__ void __launch_bounds__(kThreads)
exact_cc_kernel(const uint8_t* __restrict__ img, uint32_t W, uint32_t H,
                const uint8_t* __restrict__ planes, uint32_t tpitch, uint32_t w, uint32_t h,
                const unsigned long long* __restrict__ tss_ptr,
                const unsigned long long* __restrict__ sat,  // unmasked only
                uint32_t Wo, uint32_t Ho, int method, int precision, float* __restrict__ out) {
  using P = Planes<kVar>;
  constexpr int RY = P::RY, TY = 8 * RY, NI = P::NI, NT = P::NT, NP = P::NP;
  constexpr int kImgRows = TY + kDYC - 1;
  __shared__ __align__(16) uint8_t s_tpl[NT][kDYC][kDXC];
  __shared__ __align__(16) uint8_t s_img[NI][kImgRows][kImgPitch];

  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const uint32_t ox0 = blockIdx.x * kTX, oy0 = blockIdx.y * TY;
  const size_t tplane = (size_t)tpitch * h;

  unsigned long long X[RY][4], Y[RY][4];
#pragma unroll
  for (int j = 0; j < RY; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) X[j][i] = Y[j][i] = 0ull;

  for (uint32_t cy = 0; cy < h; cy += kDYC) {
    const int dyc = (int)min((uint32_t)kDYC, h - cy);
    for (uint32_t cx = 0; cx < w; cx += kDXC) {
      const int dxc = (int)min((uint32_t)kDXC, w - cx);
      const int ngrp = (dxc + 15) >> 4;
      __syncthreads();
      // stage template planes: kDYC x kDXC per plane, 16-byte loads
      for (int k = threadIdx.x; k < NT * kDYC * (kDXC / 16); k += kThreads) {
        const int p = k / (kDYC * (kDXC / 16));
        const int r = (k / (kDXC / 16)) % kDYC;
        const int c = (k % (kDXC / 16)) * 16;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < dyc && cx + c < tpitch)
          v = *reinterpret_cast<const uint4*>(planes + p * tplane + (size_t)(cy + r) * tpitch + cx + c);
        *reinterpret_cast<uint4*>(&s_tpl[p][r][c]) = v;
      }
      // stage image rows (and the byte planes of I^2 for masked variants)
      for (int k = threadIdx.x; k < kImgRows * kImgPitch; k += kThreads) {
        const int r = k / kImgPitch, c = k % kImgPitch;
        const uint32_t gy = oy0 + cy + r, gx = ox0 + cx + c;
        uint32_t v = 0;
        if (gy < H && gx < W) v = img[(size_t)gy * W + gx];
        s_img[0][r][c] = (uint8_t)v;
        if constexpr (NI == 3) {
          const uint32_t sq = v * v;
          s_img[1][r][c] = (uint8_t)sq;
          s_img[2][r][c] = (uint8_t)(sq >> 8);
        }
      }
      __syncthreads();

      uint32_t acc[NP][RY][4];
#pragma unroll
      for (int q = 0; q < NP; ++q)
#pragma unroll
        for (int j = 0; j < RY; ++j)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[q][j][i] = 0u;

      for (int rr = 0; rr < RY + dyc - 1; ++rr) {
        const int srow = ty * RY + rr;
        for (int g = 0; g < ngrp; ++g) {
          uint32_t sh[NI][4][4];
#pragma unroll
          for (int p = 0; p < NI; ++p) {
            const uint32_t* wp = reinterpret_cast<const uint32_t*>(&s_img[p][srow][4 * tx + 16 * g]);
            uint32_t wv[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) wv[k] = wp[k];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              sh[p][c][0] = wv[c];
              sh[p][c][1] = funnel_bytes<1>(wv[c], wv[c + 1]);
              sh[p][c][2] = funnel_bytes<2>(wv[c], wv[c + 1]);
              sh[p][c][3] = funnel_bytes<3>(wv[c], wv[c + 1]);
            }
          }
#pragma unroll
          for (int j = 0; j < RY; ++j) {
            const int dy = rr - j;
            if (dy < 0 || dy >= dyc) continue;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
              int ip, tp;
              pair_planes(kVar, q, ip, tp);
              const uint4 t4 = *reinterpret_cast<const uint4*>(&s_tpl[tp][dy][16 * g]);
              const uint32_t tw[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
              for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[q][j][i] = dp4a_u8(sh[ip][c][i], tw[c], acc[q][j][i]);
            }
          }
        }
      }
      // fold the chunk sums into the exact u64 totals
#pragma unroll
      for (int j = 0; j < RY; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if constexpr (kVar == 0) {
            X[j][i] += acc[0][j][i];
          } else if constexpr (kVar == 1) {
            X[j][i] += acc[0][j][i];
            Y[j][i] += (unsigned long long)acc[1][j][i] + ((unsigned long long)acc[2][j][i] << 8);
          } else {
            X[j][i] += (unsigned long long)acc[0][j][i] + ((unsigned long long)acc[1][j][i] << 8) +
                       ((unsigned long long)acc[2][j][i] << 16);
            Y[j][i] += (unsigned long long)acc[3][j][i] +
                       (((unsigned long long)acc[4][j][i] + acc[5][j][i]) << 8) +
                       ((unsigned long long)acc[6][j][i] << 16);
          }
        }
    }
  }

  // epilogue: method formula, one rounding to f32
  const unsigned long long tss = *tss_ptr;
  const size_t spitch = (size_t)W + 1;
#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const uint32_t y = oy0 + ty * RY + j;
    if (y >= Ho) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t x = ox0 + 4 * tx + i;
      if (x >= Wo) continue;
      unsigned long long Yv = Y[j][i];
      if constexpr (kVar == 0) {
        if (method != kCcorr) {
          const unsigned long long* top = sat + (size_t)y * spitch;
          const unsigned long long* bot = sat + (size_t)(y + h) * spitch;
          Yv = bot[x + w] - top[x + w] - bot[x] + top[x];
        }
      }
      out[(size_t)y * Wo + x] = finish_score(method, precision, X[j][i], Yv, tss);
    }
  }
}

template <int kVar>
cudaError_t launch_variant(const MatchArgs& a, const uint8_t* planes, const unsigned long long* tss,
                           const unsigned long long* sat) {
  const uint32_t Wo = a.W - a.w + 1, Ho = a.H - a.h + 1;
  constexpr int TY = 8 * Planes<kVar>::RY;
  const dim3 grid((Wo + kTX - 1) / kTX, (Ho + TY - 1) / TY);
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  timer_begin(a.timer, kKernelExactCC, a.stream);
  exact_cc_kernel<kVar><<<grid, kThreads, 0, a.stream>>>(
      a.img, a.W, a.H, planes, (uint32_t)template_pitch(a.w), a.w, a.h, tss, sat, Wo, Ho, a.method,
      a.precision, a.out);
  count_launch(kKernelExactCC);
  timer_end(a.timer, a.stream);
  return cudaGetLastError();
}

bool needs_integral(const MatchArgs& a) { return !a.mask && a.method != kCcorr; }

}  // namespace

size_t exact_cc_scratch_bytes(const MatchArgs& a) {
  size_t b = prep_scratch_bytes(a);
  if (needs_integral(a)) b += integral_bytes(a.W, a.H);
  return b;
}

cudaError_t launch_exact_cc(const MatchArgs& a, void* scratch) {
  uint8_t* base = static_cast<uint8_t*>(scratch);
  const size_t planes_bytes = prep_scratch_bytes(a) - 256;
  uint8_t* planes = base;
  unsigned long long* tss = reinterpret_cast<unsigned long long*>(base + planes_bytes);
  unsigned long long* sat = nullptr;
  cudaError_t e = launch_prep(a, planes, tss);
  if (e != cudaSuccess) return e;
  if (needs_integral(a)) {
    sat = reinterpret_cast<unsigned long long*>(base + prep_scratch_bytes(a));
    e = launch_integral_squared(a.img, a.W, a.H, sat, a.stream);
    if (e != cudaSuccess) return e;
  }
  if (!a.mask) return launch_variant<0>(a, planes, tss, sat);
  if (a.mask_binary) return launch_variant<1>(a, planes, tss, sat);
  return launch_variant<2>(a, planes, tss, sat);
}

}  // namespace ipb
