// tm_noalloc.cu -- a template-matching entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: a plug-in inside a host application
// that owns the whole device-memory budget, a latency-critical loop in which
// cudaMalloc/cudaFree would stall or synchronise the device, or code that must
// not meet an out-of-memory failure after start-up. For them,
// ipb_match_template_device_noalloc runs the CUDA-core kernels of
// ipb_match_template_device (never the tensor-core kernel, whose shapes it
// therefore runs slower, with the same scores), and its scratch memory (template planes, the
// template constant and the u64 integral image of I^2) lives in one fixed
// array compiled into this library instead of a buffer obtained at run time.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes
// (16 MiB); every GPU that loads the library holds it until the process exits.
// Host code cannot use the array's name as a device address, so the first call
// on each device looks the address up with cudaGetSymbolAddress (with that
// device current) and caches it; make that first call before any stream
// capture. The cached address is not looked up again, so calls after a
// cudaDeviceReset of that device are not supported. All calls share the one array and it keeps whatever the last call
// left there: the kernels clear what must start at zero on every call, and two
// calls that overlap on the GPU (different streams, or different host threads
// on the same device) race on it, so callers must order them.
#include <mutex>
#include <string>

#include "tm_common.cuh"
#include "tm_internal.h"

#define IPB_API extern "C" __attribute__((visibility("default")))

namespace ipb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `dev` (which must be current).
int scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      const std::string msg = std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e);
      return report_error(IPB_ERR_CUDA, msg.c_str());
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return IPB_OK;
}

}  // namespace
}  // namespace ipb

using namespace ipb;

IPB_API ipb_status ipb_match_template_device_noalloc(const uint8_t* d_image, uint32_t W, uint32_t H,
                                                     const uint8_t* d_tpl, uint32_t w, uint32_t h,
                                                     const uint8_t* d_mask, uint32_t mw, uint32_t mh,
                                                     int mask_is_binary, int method, int precision,
                                                     float* d_out, void* stream) {
  // the reference's assertions, in its order (src/template_matching.rs:433-437, :395-402)
  if (d_mask && (mw != w || mh != h))
    return (ipb_status)report_error(IPB_ERR_MASK_SIZE, "the template and mask must be the same size");
  if (W < w)
    return (ipb_status)report_error(IPB_ERR_TEMPLATE_WIDTH,
                                    "image width must be greater than or equal to template width");
  if (H < h)
    return (ipb_status)report_error(IPB_ERR_TEMPLATE_HEIGHT,
                                    "image height must be greater than or equal to template height");
  if (method < 0 || method > 3)
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "unknown MatchTemplateMethod");
  if (precision < 0 || precision > 2)
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "unknown precision");
  if ((!d_image && (size_t)W * H) || (!d_tpl && (size_t)w * h) || !d_out)
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "null buffer");

  MatchArgs a{d_image, W, H, d_tpl, w, h, d_mask, d_mask && mask_is_binary != 0, method, precision,
              d_out, static_cast<cudaStream_t>(stream)};
  const size_t need = precision == IPB_PRECISION_REFERENCE_F32 ? reference_scratch_bytes(a)
                                                               : exact_cc_scratch_bytes(a);
  if (w != 0 && h != 0 && need > kNoAllocScratchBytes) {
    const std::string msg = "ipb_match_template_device_noalloc: this problem needs " +
                            std::to_string(need) + " bytes of scratch, above the fixed maximum of " +
                            std::to_string(kNoAllocScratchBytes) +
                            " bytes; use ipb_match_template_device";
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, msg.c_str());
  }

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (ipb_status)report_error(IPB_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return (ipb_status)report_error(IPB_ERR_INVALID_ARGUMENT, "device index out of range");
  int major = 0;
  e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e != cudaSuccess) return (ipb_status)report_error(IPB_ERR_CUDA, cudaGetErrorString(e));
  if (major != 10)
    return (ipb_status)report_error(IPB_ERR_NO_DEVICE, "imageproc_b200 needs an sm_100 (B200) device");

  if (w == 0 || h == 0) {
    // empty window: every score is 0 (the walk never runs, :410-416)
    e = cudaMemsetAsync(d_out, 0, (size_t)(W - w + 1) * (H - h + 1) * sizeof(float), a.stream);
    return e == cudaSuccess ? IPB_OK : (ipb_status)report_error(IPB_ERR_CUDA, cudaGetErrorString(e));
  }
  void* scratch = nullptr;
  const int st = scratch_address(dev, &scratch);
  if (st != IPB_OK) return (ipb_status)st;
  e = precision == IPB_PRECISION_REFERENCE_F32 ? launch_reference(a, scratch) : launch_exact_cc(a, scratch);
  if (e != cudaSuccess) return (ipb_status)report_error(IPB_ERR_CUDA, cudaGetErrorString(e));
  return IPB_OK;
}
