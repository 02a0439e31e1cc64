// tm_conv_tc.cu -- the proposal network's 3x3 32 -> 32 convolution on the
// 5th-generation tensor cores (tcgen05.mma kind::f16: bf16 operands from
// shared memory, fp32 accumulators in tensor memory).
//
// Formulation (implicit GEMM per output row segment): a tile is one output
// row y of one image and 128 consecutive pixels x0 .. x0 + 127 (M = 128 =
// tensor-memory lanes), all 32 output channels (N = 32), and K = 9 taps x 32
// input channels = 18 MMAs of K = 16. The A operand of tap (ky, kx) is input
// row y + ky - 1 at pixels x0 + kx - 1 .. : the staged row, in the canonical
// no-swizzle K-major layout (for each 8-channel chunk, pixels 16 bytes apart),
// started kx pixels (16 * kx bytes) later, so one staged row serves all three
// kx taps. B is the tap's weights [co][ci], resident for the CTA's life.
//
// A CTA walks a band of output rows of one 128-pixel column segment, so each
// input row is loaded once and used by three tiles: a ring of four staged
// rows, filled by a loader warp with cp.async (zero fill outside the image),
// an MMA warp whose elected lane issues a tile's 18 MMAs into one of two
// accumulators, and four epilogue warps (one per tensor-memory lane quadrant)
// that add the bias, apply the ReLU, round to bf16 and store the row-chunked
// activations. mbarriers hand rows and accumulators between the roles; every
// wait is bounded and a wait that runs out sets the error word.
#include "imageproc_b200.h"
#include "tm_internal.h"
#include "tm_learned.cuh"
#include "tm_sm100.cuh"

namespace ipb {
namespace learned {
namespace {

using namespace sm100;

constexpr int kSeg = 128;                 // output pixels per tile (tensor-memory lanes)
constexpr int kRowPx = 136;               // staged pixels per row: kSeg + 2 halo, padded to 8
constexpr int kChunkBytes = kRowPx * 16;  // one 8-channel chunk of a staged row (2176 B)
constexpr int kRowBytes = kChunks * kChunkBytes;  // 8704 B
constexpr int kRing = 4;                  // staged input rows
constexpr int kWBytes = 9 * kChunks * kC * 16;    // 18432 B of weights
constexpr int kThreadsTc = 192;           // warp 0 MMA, warp 1 loader, warps 2..5 epilogue
constexpr uint32_t kTmemColsTc = 64;      // two accumulators of 32 columns

struct TcSmemLayout {
  static constexpr uint32_t w = 0;
  static constexpr uint32_t ring = kWBytes;
  static constexpr uint32_t bars = ring + kRing * kRowBytes;   // 13 mbarriers
  static constexpr uint32_t misc = bars + 16 * 8;              // tmem address, error flag
  static constexpr uint32_t bias = misc + 16;                  // 32 floats
  static constexpr uint32_t total = bias + kC * 4;
};

// instruction descriptor of kind::f16: bf16 A and B, fp32 D, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t M, uint32_t N) {
  return (1u << 4)            // D format: f32
         | (1u << 7)          // A format: bf16
         | (1u << 10)         // B format: bf16
         | ((N >> 3) << 17)   // N / 8
         | ((M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
}

__device__ __forceinline__ uint16_t bf16_rn(float f) {
  uint32_t u = __float_as_uint(f);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

struct TcArgs {
  const uint4* in;
  uint4* out;
  const uint16_t* wt;   // [tap][co][ci] bf16
  const float* bias;    // [32]
  int relu;
  uint32_t H, W, band;  // rows per CTA
  unsigned long long wait_ns;
  uint32_t stall;       // pipeline_stall() at launch
  unsigned int* err;    // error word or null
  unsigned int tag;
  const uint4* mask;    // or null: keeps an output bf16 only where this activation is > 0 (ReLU')
};

__global__ void __launch_bounds__(kThreadsTc) conv_tc_kernel(const TcArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t* row_full = reinterpret_cast<uint64_t*>(smem + TcSmemLayout::bars);
  uint64_t* row_empty = row_full + kRing;
  uint64_t* acc_full = row_empty + kRing;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + TcSmemLayout::misc);
  volatile uint32_t* s_err = s_tmem + 1;
  float* s_bias = reinterpret_cast<float*>(smem + TcSmemLayout::bias);

  const uint32_t n = blockIdx.z;
  const uint32_t x0 = blockIdx.x * kSeg;
  const uint32_t yb = blockIdx.y * a.band;
  const uint32_t ntiles = yb < a.H ? min(a.band, a.H - yb) : 0u;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // weights: [tap][chunk][co] 16-byte units (K-major B per tap and chunk)
  for (uint32_t i = threadIdx.x; i < 9u * kC * kChunks; i += kThreadsTc) {
    const uint32_t c = i & 3u, row = i >> 2, tap = row / kC, co = row % kC;
    reinterpret_cast<uint4*>(smem + TcSmemLayout::w)[(tap * kChunks + c) * kC + co] =
        reinterpret_cast<const uint4*>(a.wt)[i];
  }
  if (threadIdx.x < kC) s_bias[threadIdx.x] = a.bias ? a.bias[threadIdx.x] : 0.f;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kRing; ++s) {
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
  fence_proxy_async_smem();  // the weights are read by the tensor cores
  if (warp == 0) {
    tmem_alloc(s_tmem, kTmemColsTc);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const unsigned long long deadline = global_ns() + a.wait_ns;
  const uint32_t ring0 = smem_u32(smem + TcSmemLayout::ring);
  const uint32_t w0 = smem_u32(smem + TcSmemLayout::w);

  if (warp == 1) {
    // loader: input rows yb - 1 .. yb + ntiles (index i = row - yb + 1)
    const uint32_t nrows = ntiles ? ntiles + 2 : 0u;
    for (uint32_t i = 0; i < nrows; ++i) {
      const uint32_t s = i % kRing, u = i / kRing;
      if (u > 0 && !mbar_wait(&row_empty[s], (u - 1) & 1u, deadline)) {
        *s_err = 1;
        break;
      }
      const int y = (int)yb - 1 + (int)i;
      const bool row_ok = y >= 0 && y < (int)a.H;
      const uint32_t dst0 = ring0 + s * kRowBytes;
      for (uint32_t j = lane; j < (uint32_t)(kChunks * (kSeg + 2)); j += 32) {
        const uint32_t c = j / (kSeg + 2), px = j % (kSeg + 2);
        const int x = (int)x0 - 1 + (int)px;
        const bool ok = row_ok && x >= 0 && x < (int)a.W;
        const uint4* src = ok ? a.in + ((((size_t)n * a.H + y) * kChunks + c) * a.W + x) : a.in;
        cp_async16_zfill(dst0 + c * kChunkBytes + px * 16, src, ok ? 16u : 0u);
      }
      cp_async_commit_wait();
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&row_full[s]);
    }
  } else if (warp == 0) {
    // MMA issue: tile k reads staged rows k, k + 1, k + 2 (input rows y - 1 .. y + 1)
    constexpr uint32_t idesc = idesc_bf16_f32(kSeg, kC);
    const bool leader = elect_one();
    // test hook: a wait on the drain barrier, which nothing arrives at before the end
    if (a.stall && !__all_sync(0xffffffffu, mbar_wait(drain, 0, deadline))) *s_err = 1;
    for (uint32_t k = 0; k < ntiles && !*s_err; ++k) {
      bool ok = true;
      for (uint32_t j = 0; j < 3 && ok; ++j) ok = mbar_wait(&row_full[(k + j) % kRing], ((k + j) / kRing) & 1u, deadline);
      const uint32_t b = k & 1u, v = k >> 1;
      if (ok && v > 0) ok = mbar_wait(&acc_empty[b], (v - 1) & 1u, deadline);
      if (!__all_sync(0xffffffffu, ok)) {
        *s_err = 1;
        break;
      }
      tc_fence_after();
      if (leader) {
        const uint32_t d = tmem + b * kC;
#pragma unroll
        for (uint32_t tap = 0; tap < 9; ++tap) {
          const uint32_t ky = tap / 3, kx = tap % 3;
          const uint32_t arow = ring0 + ((k + ky) % kRing) * kRowBytes + kx * 16;
#pragma unroll
          for (uint32_t js = 0; js < 2; ++js) {
            const uint64_t ad = smem_desc_noswizzle(arow + 2 * js * kChunkBytes, kChunkBytes, 128);
            const uint64_t bd = smem_desc_noswizzle(w0 + (tap * kChunks + 2 * js) * kC * 16, kC * 16, 128);
            mma_bf16_ss(d, ad, bd, idesc, (tap | js) != 0);
          }
        }
        mma_commit(&acc_full[b]);
        mma_commit(&row_empty[k % kRing]);  // staged row k is not read again
      }
      __syncwarp();
    }
  } else {
    // epilogue: warp's lane quadrant q, pixel x0 + 32 q + lane
    const uint32_t q = warp & 3;
    const uint32_t x = x0 + 32 * q + lane;
    for (uint32_t k = 0; k < ntiles; ++k) {
      const uint32_t b = k & 1u, v = k >> 1;
      if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], v & 1u, deadline))) {
        *s_err = 1;
        break;
      }
      tc_fence_after();
      uint32_t r[32];
      tmem_ld32(tmem_addr(tmem, 32 * q, b * kC), r);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
      if (x < a.W) {
        const uint32_t y = yb + k;
        uint4* dst = a.out + (((size_t)n * a.H + y) * kChunks) * a.W + x;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
          uint32_t pk[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            float lo = __uint_as_float(r[8 * c + 2 * e]) + s_bias[8 * c + 2 * e];
            float hi = __uint_as_float(r[8 * c + 2 * e + 1]) + s_bias[8 * c + 2 * e + 1];
            if (a.relu) {
              lo = lo > 0.f ? lo : 0.f;
              hi = hi > 0.f ? hi : 0.f;
            }
            pk[e] = (uint32_t)bf16_rn(lo) | ((uint32_t)bf16_rn(hi) << 16);
          }
          if (a.mask) {
            // the data gradient: times ReLU'(Z) = [A > 0] of the layer's activation
            const uint4 mk = a.mask[(((size_t)n * a.H + y) * kChunks + c) * a.W + x];
            const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const bool plo = (int16_t)(mw[e] & 0xFFFFu) > 0, phi = (int16_t)(mw[e] >> 16) > 0;
              pk[e] &= (plo ? 0x0000FFFFu : 0u) | (phi ? 0xFFFF0000u : 0u);
            }
          }
          dst[(size_t)c * a.W] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
      }
    }
  }

  // every tensor-core operation of this CTA completes before its tensor
  // memory is freed (this wait keeps the full default budget)
  __syncthreads();
  if (warp == 0) {
    mma_commit_warp(drain);
    if (!mbar_wait(drain, 0, global_ns() + kDefaultWaitNs)) *s_err = 1;
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemColsTc);
  }
  if (threadIdx.x == 0 && *s_err && a.err) atomicMax(a.err, a.tag);
}

}  // namespace

cudaError_t launch_conv_tc(const uint4* in, uint32_t n, uint32_t H, uint32_t W, const uint16_t* wt,
                           const float* bias, int relu, uint4* out, unsigned int* err, unsigned int tag,
                           cudaStream_t s, const uint4* mask) {
  if (n == 0 || H == 0 || W == 0) return cudaSuccess;
  static PerDeviceOnce attr;
  cudaError_t e = attr.run([] {
    return cudaFuncSetAttribute(conv_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)TcSmemLayout::total);
  });
  if (e != cudaSuccess) return e;
  const uint32_t segs = (W + kSeg - 1) / kSeg;
  // about two CTAs per SM over the whole launch, at least 4 rows per band
  const uint64_t want = 2ull * (uint64_t)device_sm_count();
  uint64_t bands = want / ((uint64_t)segs * n);
  if (bands < 1) bands = 1;
  uint32_t band = (uint32_t)((H + bands - 1) / bands);
  if (band < 4) band = 4;
  if (band > H) band = H;
  const dim3 grid(segs, (H + band - 1) / band, n);
  TcArgs args{in, out, wt, bias, relu, H, W, band, pipeline_wait_ns(), pipeline_stall() ? 1u : 0u, err, tag, mask};
  conv_tc_kernel<<<grid, kThreadsTc, TcSmemLayout::total, s>>>(args);
  count_launch(kKernelLearned);
  return cudaGetLastError();
}

}  // namespace learned
}  // namespace ipb
