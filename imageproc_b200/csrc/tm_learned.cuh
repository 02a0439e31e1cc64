// tm_learned.cuh -- the proposal network's data layout and launchers, shared
// by the training entry points (tm_learned.cu) and the query pipeline
// (tm_propose.cu).
//
// The network (no counterpart in the reference, which scores every window):
//   D       4x4 block sums of the u8 image, (sum - 2048) / 1024          (fp32)
//   A1      bf16(relu(b1 + conv3x3(W1, D)))                1 -> 32 channels
//   A2..A4  bf16(relu(bl + conv3x3(Wl, A(l-1))))          32 -> 32
//   F       bf16(b5 + conv3x3(W5, A4))                     32 -> 32, no relu
//   G_t(o)  F of template t (48 x 48 -> 12 x 12) at (5 + oy, 5 + ox), o in {0,1}^2
//   z_t(p)  = alpha * sum_o F(p + o) . G_t(o)              (F outside = 0)
// Convolutions pad with zeros. z_t peaks at p = q + 5 when the template's
// downsampled top-left corner is at q, so a heatmap position p proposes the
// full-resolution top-left 4 (p - 5).
//
// Activation layout ("row-chunked"): image n, row y, channel chunk c (8
// channels), pixel x: one 16-byte unit of 8 bf16 at index
// ((n * H + y) * 4 + c) * W + x. A row's 8-channel chunks are contiguous runs
// of pixels, so the tensor-core operands (pixels x channels) load as 16-byte
// rows. Parameters (fp32, canonical order, IPB_PROPOSAL_NET_PARAMS values):
//   W1 [32][1][3][3], b1 [32], then for l = 2..5: Wl [32][32][3][3], bl [32].
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ipb {
namespace learned {

constexpr int kC = 32;       // channels
constexpr int kChunks = 4;   // 8-channel chunks
constexpr int kLayers = 5;
constexpr int kTpl = 48;     // template side (pixels)
constexpr int kTplDs = 12;   // downsampled template side
constexpr int kCentre = 5;   // first centre position of the 2x2 template embedding
constexpr int kEmb = 4 * kC; // embedding length: 4 offsets x 32 channels
constexpr float kAlpha = 0.125f;
constexpr int kParams = kC * 9 + kC + (kLayers - 1) * (kC * kC * 9 + kC);  // 37312

// offsets into the parameter vector
__host__ __device__ constexpr int w_off(int l) { return l == 0 ? 0 : kC * 9 + kC + (l - 1) * (kC * kC * 9 + kC); }
__host__ __device__ constexpr int b_off(int l) { return l == 0 ? kC * 9 : w_off(l) + kC * kC * 9; }

inline size_t act_units(uint32_t n, uint32_t H, uint32_t W) { return (size_t)n * H * kChunks * W; }

// bf16 weights of layers 2..5 in the tensor-core layouts: forward [tap][co][ci]
// and, for the data gradient, flipped taps with the channel roles swapped
// [8 - tap][ci][co].
struct PackedWeights {
  uint16_t* fwd;   // 4 x 9 x 32 x 32
  uint16_t* bwd;   // 4 x 9 x 32 x 32
  float* w1;       // 32 x 9, bf16-rounded values
  float* bias;     // 5 x 32
};

cudaError_t launch_pack_weights(const float* params, PackedWeights pw, cudaStream_t s);
// layer 1 from the u8 image (downsampled on the fly)
cudaError_t launch_conv1(const uint8_t* img, uint32_t n, uint32_t h, uint32_t w, const float* w1, const float* b1,
                         uint4* out, cudaStream_t s);
// one 3x3 32 -> 32 convolution on bf16 tensor cores (mma.sync), fp32
// accumulation: out = bf16(act(bias + conv(wt, in))) [* (mask > 0)]
cudaError_t launch_conv_mma(const uint4* in, uint32_t n, uint32_t H, uint32_t W, const uint16_t* wt,
                            const float* bias, int relu, const uint4* mask, uint4* out, cudaStream_t s);
// the same convolution on tcgen05 (kind::f16, accumulators in tensor memory):
// out = bf16(act(bias + conv(wt, in))), times [mask > 0] when mask is not null
// (the data gradient of a ReLU layer); a bounded wait that runs out stores
// `tag` into *err (when err is not null)
cudaError_t launch_conv_tc(const uint4* in, uint32_t n, uint32_t H, uint32_t W, const uint16_t* wt,
                           const float* bias, int relu, uint4* out, unsigned int* err, unsigned int tag,
                           cudaStream_t s, const uint4* mask = nullptr);
// IPB_LEARNED_KERNELS=mma: the network's 32-channel convolutions and heatmap
// on the mma.sync kernels instead of tcgen05 (same arithmetic: bf16 operands,
// fp32 accumulation), in queries and in training; for testing and measurement.
bool learned_use_mma();
// the trunk: conv1 + four tensor-core layers; acts (4 buffers) keeps A1..A4
// when not null (training), otherwise ping-pong buffers a/b are used.
// kernel: 0 = tcgen05 (launch_conv_tc), 1 = mma.sync (launch_conv_mma)
cudaError_t launch_trunk(const uint8_t* img, uint32_t n, uint32_t h, uint32_t w, const PackedWeights& pw,
                         uint4* const* acts, uint4* tmp_a, uint4* tmp_b, uint4* F, cudaStream_t s,
                         int kernel = 1, unsigned int* err = nullptr, unsigned int tag = 0);
// heatmap cell maxima on tcgen05: cells[t][cy][cx] = max over the cell's 8 x 8
// positions of (order key of z_t << 32) | ~position (gb: [4][T][32] bf16)
cudaError_t launch_head_tc(const uint4* F, uint32_t Hs, uint32_t Ws, const uint16_t* gb, uint32_t T,
                           unsigned long long* cells, unsigned int* err, unsigned int tag, cudaStream_t s);
// G[t][o * 32 + c] (fp32) from the templates' 12 x 12 feature maps
cudaError_t launch_embed(const uint4* Ft, uint32_t T, float* G, cudaStream_t s);

}  // namespace learned
}  // namespace ipb
