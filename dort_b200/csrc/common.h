// Shared host/device definitions of the dort_gpu library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/dort_gpu.h"

namespace dort_gpu {

// Thread-local message behind dort_gpu_last_error().
void set_error(const std::string& msg);
void clear_error();
int fail(int code, const std::string& msg);

#define DG_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if(e_ != cudaSuccess) {                                                  \
      return ::dort_gpu::fail(DORT_ERR_CUDA, std::string(#call " failed: ") + \
                              cudaGetErrorString(e_));                       \
    }                                                                        \
  } while(0)

// Device view of the ray-query part of a scene.
struct TraceScene {
  const uint4* nodes;   // 5 x uint4 per WideNode (bvh_build.h)
  const float4* tris;   // 3 x float4 per LeafTri
  uint32_t node_count;
  uint32_t tri_count;
};

}  // namespace dort_gpu

// Host-side scene handle behind the opaque dort_scene.
struct dort_scene {
  int device = 0;
  dort_gpu::TraceScene trace{};
  uint32_t depth = 0;
  uint32_t tri_count = 0;
  uint32_t emissive_count = 0;
  size_t device_bytes = 0;
  double build_ms = 0.0;
  void* d_nodes = nullptr;
  void* d_tris = nullptr;
  uint32_t* d_work = nullptr;          // persistent-kernel work counters (scratch)
  // staging for the host-pointer entry points (grow-only)
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
};
