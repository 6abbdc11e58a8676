// Scene creation / destruction and the error plumbing of the C ABI.
#include <chrono>
#include <cstring>
#include <string>

#include "bvh_build.h"
#include "common.h"

namespace dort_gpu {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" const char* dort_gpu_last_error(void) { return g_last_error.c_str(); }

extern "C" int dort_gpu_abi_version(void) { return DORT_GPU_ABI_VERSION; }

static void scene_free_device(dort_scene* s) {
  if(s->d_nodes) { cudaFree(s->d_nodes); }
  if(s->d_tris) { cudaFree(s->d_tris); }
  if(s->d_work) { cudaFree(s->d_work); }
  if(s->d_stage) { cudaFree(s->d_stage); }
  s->d_nodes = s->d_tris = s->d_stage = nullptr;
  s->d_work = nullptr;
}

extern "C" int dort_gpu_scene_create(const dort_scene_desc* desc, dort_scene** out_scene) {
  clear_error();
  if(!desc || !out_scene) { return fail(DORT_ERR_INVALID, "null argument"); }
  *out_scene = nullptr;
  if(desc->struct_size != sizeof(dort_scene_desc)) {
    return fail(DORT_ERR_INVALID, "dort_scene_desc.struct_size mismatch (ABI version)");
  }
  if(desc->tri_count > 0 && (!desc->verts || !desc->tris)) {
    return fail(DORT_ERR_INVALID, "verts and tris are required when tri_count > 0");
  }
  if(desc->tri_count > (1u << 30)) {
    return fail(DORT_ERR_INVALID, "tri_count exceeds 2^30");
  }

  auto t0 = std::chrono::steady_clock::now();
  BuildOptions opts;
  opts.width = desc->bvh_width ? desc->bvh_width : 8;
  WideBvh bvh;
  std::string err;
  if(!build_wide_bvh(desc->verts, desc->vert_count, desc->tris, desc->tri_count,
                     opts, bvh, err)) {
    return fail(DORT_ERR_INVALID, err);
  }
  auto t1 = std::chrono::steady_clock::now();

  dort_scene* s = new dort_scene();
  cudaGetDevice(&s->device);
  s->tri_count = desc->tri_count;
  s->depth = bvh.depth;
  s->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

  size_t node_bytes = bvh.nodes.size() * sizeof(WideNode);
  size_t tri_bytes = bvh.tris.size() * sizeof(LeafTri);
  auto cleanup_fail = [&](int code, const std::string& msg) {
    scene_free_device(s);
    delete s;
    return fail(code, msg);
  };
  if(node_bytes) {
    if(cudaMalloc(&s->d_nodes, node_bytes) != cudaSuccess) {
      cudaGetLastError();
      return cleanup_fail(DORT_ERR_OOM, "cudaMalloc of BVH nodes failed");
    }
    if(cudaMemcpy(s->d_nodes, bvh.nodes.data(), node_bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      return cleanup_fail(DORT_ERR_CUDA, "copy of BVH nodes failed");
    }
  }
  if(tri_bytes) {
    if(cudaMalloc(&s->d_tris, tri_bytes) != cudaSuccess) {
      cudaGetLastError();
      return cleanup_fail(DORT_ERR_OOM, "cudaMalloc of triangles failed");
    }
    if(cudaMemcpy(s->d_tris, bvh.tris.data(), tri_bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      return cleanup_fail(DORT_ERR_CUDA, "copy of triangles failed");
    }
  }
  if(cudaMalloc(&s->d_work, 64 * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return cleanup_fail(DORT_ERR_OOM, "cudaMalloc of work counters failed");
  }
  s->trace.nodes = static_cast<const uint4*>(s->d_nodes);
  s->trace.tris = static_cast<const float4*>(s->d_tris);
  s->trace.node_count = uint32_t(bvh.nodes.size());
  s->trace.tri_count = uint32_t(bvh.tris.size());
  s->device_bytes = node_bytes + tri_bytes + 64 * sizeof(uint32_t);
  *out_scene = s;
  return DORT_OK;
}

extern "C" int dort_gpu_scene_destroy(dort_scene* scene) {
  clear_error();
  if(!scene) { return DORT_OK; }
  scene_free_device(scene);
  delete scene;
  return DORT_OK;
}

extern "C" int dort_gpu_scene_stats(const dort_scene* s, double out[8]) {
  clear_error();
  if(!s || !out) { return fail(DORT_ERR_INVALID, "null argument"); }
  out[0] = s->trace.node_count;
  out[1] = s->depth;
  out[2] = s->tri_count;
  out[3] = s->emissive_count;
  out[4] = double(s->device_bytes);
  out[5] = s->build_ms;
  out[6] = 0.0;
  out[7] = 0.0;
  return DORT_OK;
}
