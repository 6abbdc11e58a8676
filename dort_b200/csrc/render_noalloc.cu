// dort_gpu_render_device_noalloc: the per-pixel path tracer for callers that
// must not allocate GPU memory during a render.
//
// Some callers of a renderer cannot let it call cudaMalloc / cudaFree while
// they run: a host application that owns every device allocation under a
// fixed budget (a plugin inside another program's render loop, whose memory
// manager accounts for all device memory), or a real-time loop that cannot
// afford the device-wide synchronisation cudaFree implies.
// dort_gpu_render_device grows a per-scene scratch buffer on demand; this
// variant keeps its scratch in a fixed array that the library holds on every
// GPU it is loaded on, so a call only launches kernels and clears part of
// that array.
//
// The scratch holds the per-(slice, pixel) partial sums of the megakernel and
// two counters, kNoAllocScratchBytes in total, which caps the image at
// kNoAllocMaxPixels pixels; larger images are rejected with DORT_ERR_INVALID.
// Every call on a device shares the one array and finds the previous call's
// contents in it: the counters are cleared at the start of each call and the
// partial sums are fully overwritten by the kernel before they are read.  Two
// calls whose work overlaps on the GPU (different streams, or different
// threads without ordering) race on the array and corrupt each other's image;
// callers serialise them.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current) and keeps
// it; make that first call before any stream capture begins.  A process that
// calls cudaDeviceReset must not call this entry point on that device
// afterwards: the kept address belonged to the destroyed context.
#include <algorithm>
#include <mutex>
#include <string>

#include "common.h"
#include "launch_plan.h"
#include "pt_scene.h"

namespace dort_gpu {

// The megakernel (both instantiations) and its resolve step (pt_render.cu).
template<bool G>
__global__ void pt_megakernel(PtScene sc, PtParams pp, uint32_t slices, uint32_t spp_per_slice,
                              uint32_t per_slice, float4* __restrict__ partial,
                              unsigned long long* __restrict__ ray_count);
__global__ void pt_resolve(const float4* __restrict__ partial, uint32_t slices, uint32_t npix,
                           float* __restrict__ out_rgb, unsigned long long* __restrict__ kept);
bool make_params(const dort_render_params* rp, PtParams& pp, std::string& err);

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;   // 16 MiB per GPU
constexpr size_t kNoAllocHeader = 256;                       // counters
constexpr size_t kNoAllocMaxPixels = (kNoAllocScratchBytes - kNoAllocHeader) / sizeof(float4);
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once).
static int noalloc_scratch(void** out) {
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  if(dev < 0 || dev >= kNoAllocMaxDevices) {
    return fail(DORT_ERR_UNSUPPORTED, "device index out of range for the no-alloc scratch");
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if(!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if(e != cudaSuccess || !p) {
      return fail(DORT_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch "
                                             "failed: ") + cudaGetErrorString(e));
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return DORT_OK;
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_render_device_noalloc(dort_scene* scene,
                                              const dort_render_params* params,
                                              float* d_out_rgb, void* stream) try {
  clear_error();
  if(!scene || !params || !d_out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(pp.renderer != RENDERER_PT) {
    return fail(DORT_ERR_UNSUPPORTED, "dort_gpu_render_device_noalloc renders only the pt renderer");
  }
  size_t npix = size_t(pp.width) * pp.height;
  if(npix > kNoAllocMaxPixels) {
    return fail(DORT_ERR_INVALID, "image of " + std::to_string(npix) + " pixels exceeds the " +
                                  std::to_string(kNoAllocMaxPixels) +
                                  "-pixel limit of dort_gpu_render_device_noalloc");
  }
  // the launch shape of dort_gpu_render_device, with the slices capped so
  // that slices * pixels partial sums fit in the scratch; a scene on another
  // device is refused before anything is launched
  int dev = 0, sms = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MegaPlan plan;
  if(megakernel_plan(scene->device, dev, sms, pp.width, pp.height, pp.spp, kNoAllocMaxPixels,
                     &plan) != 0) {
    return fail(DORT_ERR_INVALID, std::string("dort_gpu_render_device_noalloc: ") + plan.why);
  }
  const uint32_t slices = plan.slices, per = plan.per, per_slice = plan.per_slice;
  if(size_t(slices) * npix > kNoAllocMaxPixels) {
    return fail(DORT_ERR_INVALID, "partial sums exceed the no-alloc scratch");
  }
  void* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if(rc != DORT_OK) { return rc; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  unsigned long long* counters = static_cast<unsigned long long*>(scratch);
  float4* partial = reinterpret_cast<float4*>(static_cast<char*>(scratch) + kNoAllocHeader);
  DG_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st));
  uint64_t threads = uint64_t(slices) * per_slice;
  const int block = 128;   // the megakernel's launch bound
  if(scene_needs_general(scene->pt, pp)) {
    pt_megakernel<true><<<uint32_t((threads + block - 1) / block), block, 0, st>>>(
        scene->pt, pp, slices, per, per_slice, partial, counters);
  } else {
    pt_megakernel<false><<<uint32_t((threads + block - 1) / block), block, 0, st>>>(
        scene->pt, pp, slices, per, per_slice, partial, counters);
  }
  DG_CUDA(cudaGetLastError());
  pt_resolve<<<uint32_t((npix + 255) / 256), 256, 0, st>>>(partial, slices, uint32_t(npix),
                                                            d_out_rgb, counters + 1);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
} DORT_ABI_CATCH
