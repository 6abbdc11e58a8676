// Shared host/device definitions of the dort_gpu library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include <vector>

#include "../../include/dort_gpu.h"
#include "pt_scene.h"

struct dort_scene;

namespace dort_gpu {

struct Wavefront;

// Thread-local message behind dort_gpu_last_error().
void set_error(const std::string& msg);
void clear_error();
int fail(int code, const std::string& msg);

// Every entry point of the C ABI ends in a function-try-block whose handler
// is DORT_ABI_CATCH: an exception (a host allocation that failed, ...)
// becomes a status code (DORT_ERR_OOM for std::bad_alloc) and never crosses
// the C ABI.
int abi_exception();
#define DORT_ABI_CATCH \
  catch(...) { return ::dort_gpu::abi_exception(); }

// DORT_OK when the scene lives on the current device, else DORT_ERR_INVALID:
// a kernel given another GPU's BVH and triangle pointers would read a peer's
// memory (or fault), so entry points check before launching.
int require_scene_device(const dort_scene* s);

// Allocation hooks.  Every device and pinned host allocation of the library
// goes through dev_alloc / host_pinned_alloc, and the host-side builders call
// alloc_checkpoint() before their large allocations; a test can make the
// n-th of these fail (dort_gpu_debug_fail_alloc) to drive the error paths
// without exhausting memory.  alloc_checkpoint throws std::bad_alloc when
// the injected failure is due.
bool alloc_injected_failure();
cudaError_t dev_alloc_bytes(void** p, size_t bytes);
cudaError_t host_pinned_alloc_bytes(void** p, size_t bytes);
void alloc_checkpoint();
template<class T>
cudaError_t dev_alloc(T** p, size_t bytes) {
  return dev_alloc_bytes(reinterpret_cast<void**>(p), bytes);
}
template<class T>
cudaError_t host_pinned_alloc(T** p, size_t bytes) {
  return host_pinned_alloc_bytes(reinterpret_cast<void**>(p), bytes);
}

#define DG_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if(e_ != cudaSuccess) {                                                  \
      return ::dort_gpu::fail(DORT_ERR_CUDA, std::string(#call " failed: ") + \
                              cudaGetErrorString(e_));                       \
    }                                                                        \
  } while(0)

}  // namespace dort_gpu

struct dort_scene;

namespace dort_gpu {

// Render scratch kept with the scene (grown on demand; pt_render.cu).
int render_scratch(dort_scene* s, size_t bytes, void** out);

// The device image of the host-pointer render entry points, kept with the
// scene (grown on demand; pt_render.cu).
int render_image_buffer(dort_scene* s, size_t bytes, float** out);

// The "lt" renderer into d_out (width * height * 3 floats) on stream st;
// d_counters[0] += rays traced, d_counters[1] += paths (lt.cu).
int launch_light_trace(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                       unsigned long long* d_counters);

// The "bdpt" renderer into d_out; counters as launch_light_trace (bdpt.cu).
int launch_bdpt(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                unsigned long long* d_counters);

}  // namespace dort_gpu

// Host-side scene handle behind the opaque dort_scene.
struct dort_scene {
  int device = 0;
  dort_gpu::TraceScene trace{};
  dort_gpu::PtScene pt{};               // device view for the path tracers
  uint32_t depth = 0;
  uint32_t tri_count = 0;
  uint32_t emissive_count = 0;
  size_t device_bytes = 0;
  double build_ms = 0.0;
  double bvh_ms = 0.0;                  // BVH build alone
  uint32_t bvh_builder = 0;             // DORT_BVH_BUILD_HOST / _DEVICE
  uint32_t bvh_iterations = 0;          // SAH levels / PLOC iterations of a device build
  std::vector<void*> allocations;       // every device buffer owned by the scene
  dort_gpu::Wavefront* wavefront = nullptr;  // wavefront queues + frame graph (lazy)
  dort_gpu::Wavefront* adj_wavefront = nullptr;  // the adjoint's backward pass (lazy)
  float* d_tri_albedo = nullptr;        // per-triangle overrides (adjoint), lazy
  float* d_tri_emission = nullptr;
  uint32_t* d_work = nullptr;           // work counters of persistent kernels (scratch)
  // render scratch (grow-only)
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  // device image of the host-pointer render entry points (grow-only)
  void* d_image = nullptr;
  size_t image_bytes = 0;
  // the adjoint's image gradient and triangle gradients (grow-only)
  void* d_adjoint = nullptr;
  size_t adjoint_bytes = 0;
  // the last backward pass: engine (0 wavefront, 1 megakernel, 2 wavefront
  // then megakernel), samples traced a second time, rays, waves
  double adjoint_stats[4] = {0.0, 0.0, 0.0, 0.0};
};
