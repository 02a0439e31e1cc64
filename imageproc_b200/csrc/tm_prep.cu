// tm_prep.cu -- template-side operand planes and the template constant TSS.
//
// The reference computes its per-template constant in `init`
// (square_sum / mult_square_sum, src/template_matching.rs:378-386). The exact
// path needs that constant as a u64 and the template-side factors of the two
// correlations as u8 planes, so that every product the kernels form is a
// u8 x u8 product (dp4a on CUDA cores, kind::i8 on the tensor cores).
#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {

int template_plane_count(const MatchArgs& a) {
  if (!a.mask) return 1;
  return a.mask_binary ? 2 : 5;
}

size_t template_pitch(uint32_t w) { return align_up(w ? w : 1, 64); }

size_t prep_scratch_bytes(const MatchArgs& a) {
  return align_up((size_t)template_plane_count(a) * a.h * template_pitch(a.w), 256) + 256;
}

// One thread per padded template byte. Planes are written for every padded
// column (zero beyond w) so the consumers can use 16-byte loads.
__global__ void prep_kernel(const uint8_t* __restrict__ tpl, const uint8_t* __restrict__ mask,
                            uint32_t w, uint32_t h, uint32_t pitch, int nplanes,
                            uint8_t* __restrict__ planes, unsigned long long* __restrict__ tss) {
  const size_t plane = (size_t)pitch * h;
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long t2 = 0;
  if (k < plane) {
    const uint32_t dy = (uint32_t)(k / pitch), dx = (uint32_t)(k % pitch);
    uint32_t t = 0, m = 0;
    if (dx < w) {
      t = tpl[(size_t)dy * w + dx];
      m = mask ? mask[(size_t)dy * w + dx] : 1u;
    }
    const uint32_t tm = t * m;
    t2 = (unsigned long long)tm * tm;
    if (nplanes == 1) {
      planes[k] = (uint8_t)t;
    } else if (nplanes == 2) {
      planes[k] = (uint8_t)tm;        // T*m (m in {0,1})
      planes[plane + k] = (uint8_t)m;  // m^2 == m
    } else {
      const uint32_t u = tm * m;       // T*m^2 < 2^24
      const uint32_t v = m * m;        // m^2 < 2^16
      planes[k] = (uint8_t)u;
      planes[plane + k] = (uint8_t)(u >> 8);
      planes[2 * plane + k] = (uint8_t)(u >> 16);
      planes[3 * plane + k] = (uint8_t)v;
      planes[4 * plane + k] = (uint8_t)(v >> 8);
    }
  }
  // warp reduction of TSS, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) t2 += __shfl_down_sync(0xffffffffu, t2, o);
  if ((threadIdx.x & 31) == 0 && t2) atomicAdd(tss, t2);
}

cudaError_t launch_prep(const MatchArgs& a, uint8_t* planes, unsigned long long* tss) {
  cudaError_t e = cudaMemsetAsync(tss, 0, sizeof(unsigned long long), a.stream);
  if (e != cudaSuccess) return e;
  const uint32_t pitch = (uint32_t)template_pitch(a.w);
  const size_t n = (size_t)pitch * a.h;
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  prep_kernel<<<blocks, threads, 0, a.stream>>>(a.tpl, a.mask, a.w, a.h, pitch,
                                                 template_plane_count(a), planes, tss);
  count_launch(kKernelPrep);
  return cudaGetLastError();
}

}  // namespace ipb
