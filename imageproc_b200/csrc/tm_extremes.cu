// tm_extremes.cu -- find_extremes as a one-launch device reduction.
//
// Reference: find_extremes (src/template_matching.rs:479-511) seeds min and
// max from pixel (0, 0) and scans in row-major order with strict < and >.
// Consequences kept here:
//   * ties resolve to the lowest linear index (first occurrence);
//   * a NaN is never taken (every comparison with it is false), except that a
//     NaN seed at (0, 0) is never replaced, so it is returned for both.
// The reduction carries (value, index) pairs and orders equal values by
// index, which reproduces the scan's choice; NaNs are excluded from the
// candidates and the seed rule is applied at the end.
//
// One launch: each block reduces a grid-stride share into a partial record;
// the last block to finish (atomic ticket) reduces the partials, writes the
// result and re-arms the ticket for the next call.
#include <cfloat>
#include <cmath>

#include "tm_common.cuh"
#include "tm_internal.h"

namespace ipb {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;

template <typename T>
__device__ __forceinline__ bool is_nan(T v) {
  if constexpr (std::is_floating_point<T>::value) return v != v;
  else return false;
}

template <typename T>
struct Cand {
  T mn, mx;
  unsigned long long imn, imx;
  int has;
};

template <typename T>
__device__ __forceinline__ void merge(Cand<T>& a, const Cand<T>& b) {
  if (!b.has) return;
  if (!a.has) { a = b; return; }
  if (b.mn < a.mn || (b.mn == a.mn && b.imn < a.imn)) { a.mn = b.mn; a.imn = b.imn; }
  if (b.mx > a.mx || (b.mx == a.mx && b.imx < a.imx)) { a.mx = b.mx; a.imx = b.imx; }
}

template <typename T>
__device__ __forceinline__ Cand<T> shfl_cand(const Cand<T>& c, int src) {
  Cand<T> o;
  o.mn = __shfl_sync(0xffffffffu, c.mn, src);
  o.mx = __shfl_sync(0xffffffffu, c.mx, src);
  o.imn = __shfl_sync(0xffffffffu, c.imn, src);
  o.imx = __shfl_sync(0xffffffffu, c.imx, src);
  o.has = __shfl_sync(0xffffffffu, c.has, src);
  return o;
}

// 8- and 16-bit values travel through the shuffles widened to 32 bits.
template <typename T> struct Wide { using type = T; };
template <> struct Wide<uint8_t> { using type = uint32_t; };
template <> struct Wide<uint16_t> { using type = uint32_t; };
template <> struct Wide<int8_t> { using type = int32_t; };
template <> struct Wide<int16_t> { using type = int32_t; };

template <typename C>
__device__ C block_reduce(C c, C* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    C other = shfl_cand(c, (lane + o) & 31);
    if (lane + o < 32) merge(c, other);
  }
  if (lane == 0) s_warp[warp] = c;
  __syncthreads();
  if (warp == 0) {
    c = lane < kThreads / 32 ? s_warp[lane] : C{};
    if (lane >= kThreads / 32) c.has = 0;
    for (int o = 16; o > 0; o >>= 1) {
      C other = shfl_cand(c, (lane + o) & 31);
      if (lane + o < 32) merge(c, other);
    }
  }
  return c;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
extremes_kernel(const T* __restrict__ data, unsigned long long n,
                Cand<typename Wide<T>::type>* __restrict__ partials, unsigned int* __restrict__ ticket,
                ExtremesResult<T>* __restrict__ result) {
  using V = typename Wide<T>::type;
  using C = Cand<V>;
  __shared__ C s_warp[kThreads / 32];
  __shared__ bool s_last;
  C c;
  c.has = 0;
  c.mn = c.mx = V(0);
  c.imn = c.imx = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * kThreads;
  for (unsigned long long k = (unsigned long long)blockIdx.x * kThreads + threadIdx.x; k < n; k += stride) {
    const T v = data[k];
    if (is_nan(v)) continue;
    const V wv = (V)v;
    if (!c.has) {
      c.mn = c.mx = wv;
      c.imn = c.imx = k;
      c.has = 1;
    } else {
      if (wv < c.mn) { c.mn = wv; c.imn = k; }  // increasing k: strict keeps the first
      if (wv > c.mx) { c.mx = wv; c.imx = k; }
    }
  }
  c = block_reduce(c, s_warp);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = c;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  C acc;
  acc.has = 0;
  acc.mn = acc.mx = V(0);
  acc.imn = acc.imx = 0;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += kThreads) {
    // other blocks' records: read through L2, never a stale L1 line
    const C* src = partials + b;
    C p;
    p.mn = __ldcg(&src->mn);
    p.mx = __ldcg(&src->mx);
    p.imn = __ldcg(&src->imn);
    p.imx = __ldcg(&src->imx);
    p.has = __ldcg(&src->has);
    merge(acc, p);
  }
  __syncthreads();
  acc = block_reduce(acc, s_warp);
  if (threadIdx.x == 0) {
    const T seed = data[0];
    ExtremesResult<T> r;
    if (is_nan(seed) || !acc.has) {
      r.max_value = r.min_value = seed;
      r.max_index = r.min_index = 0;
    } else {
      r.max_value = (T)acc.mx;
      r.min_value = (T)acc.mn;
      r.max_index = acc.imx;
      r.min_index = acc.imn;
    }
    *result = r;
    *ticket = 0u;  // re-arm for the next launch on this scratch
  }
}

}  // namespace

size_t extremes_scratch_bytes() {
  // partial records (largest element type) + ticket
  return align_up(sizeof(Cand<double>) * kMaxBlocks, 256) + 256;
}

template <typename T>
cudaError_t launch_find_extremes(const T* d, unsigned long long n, void* scratch,
                                 ExtremesResult<T>* d_result, cudaStream_t s) {
  using C = Cand<typename Wide<T>::type>;
  uint8_t* base = static_cast<uint8_t*>(scratch);
  C* partials = reinterpret_cast<C*>(base);
  unsigned int* ticket =
      reinterpret_cast<unsigned int*>(base + align_up(sizeof(Cand<double>) * kMaxBlocks, 256));
  unsigned long long blocks = (n + kThreads * 8 - 1) / (kThreads * 8);
  if (blocks < 1) blocks = 1;
  if (blocks > (unsigned long long)kMaxBlocks) blocks = kMaxBlocks;
  extremes_kernel<T><<<(unsigned)blocks, kThreads, 0, s>>>(d, n, partials, ticket, d_result);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

namespace {
__global__ void extremes_result_to_struct_kernel(const ExtremesResult<float>* r, uint32_t width,
                                                 ipb_extremes_f32* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ipb_extremes_f32 e;
  e.max_value = r->max_value;
  e.min_value = r->min_value;
  e.max_value_location_x = (uint32_t)(r->max_index % width);
  e.max_value_location_y = (uint32_t)(r->max_index / width);
  e.min_value_location_x = (uint32_t)(r->min_index % width);
  e.min_value_location_y = (uint32_t)(r->min_index / width);
  *out = e;
}
}  // namespace

cudaError_t launch_extremes_to_struct(const ExtremesResult<float>* r, uint32_t width, ipb_extremes_f32* out,
                                      cudaStream_t s) {
  extremes_result_to_struct_kernel<<<1, 32, 0, s>>>(r, width, out);
  count_launch(kKernelExtremes);
  return cudaGetLastError();
}

#define IPB_INSTANTIATE_EXTREMES(T)                                                            \
  template cudaError_t launch_find_extremes<T>(const T*, unsigned long long, void*,            \
                                               ExtremesResult<T>*, cudaStream_t);
IPB_INSTANTIATE_EXTREMES(uint8_t)
IPB_INSTANTIATE_EXTREMES(uint16_t)
IPB_INSTANTIATE_EXTREMES(uint32_t)
IPB_INSTANTIATE_EXTREMES(unsigned long long)
IPB_INSTANTIATE_EXTREMES(int8_t)
IPB_INSTANTIATE_EXTREMES(int16_t)
IPB_INSTANTIATE_EXTREMES(int32_t)
IPB_INSTANTIATE_EXTREMES(long long)
IPB_INSTANTIATE_EXTREMES(float)
IPB_INSTANTIATE_EXTREMES(double)

}  // namespace ipb
