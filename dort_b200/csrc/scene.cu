// Scene creation / destruction and the error plumbing of the C ABI.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <new>
#include <stdexcept>
#include <cstring>
#include <string>

#include "bvh_build.h"
#include "bvh_device.h"
#include "common.h"
#include "scene_build.h"
#include "wavefront.h"

namespace dort_gpu {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int abi_exception() {
  try {
    throw;
  } catch(const std::bad_alloc&) {
    return fail(DORT_ERR_OOM, "host allocation failed");
  } catch(const std::exception& e) {
    return fail(DORT_ERR_INVALID, std::string("exception: ") + e.what());
  } catch(...) {
    return fail(DORT_ERR_INVALID, "unknown exception");
  }
}

int require_scene_device(const dort_scene* s) {
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  if(s->device != dev) {
    return fail(DORT_ERR_INVALID, "scene on device " + std::to_string(s->device) +
                                  ", current device is " + std::to_string(dev));
  }
  return DORT_OK;
}

// Failure injection: the number of allocations (device, pinned host, host
// checkpoints) still allowed to succeed before one fails; negative = off.
static std::atomic<long long> g_alloc_budget{-1};

bool alloc_injected_failure() {
  long long b = g_alloc_budget.load();
  while(b >= 0) {
    if(g_alloc_budget.compare_exchange_weak(b, b - 1)) { return b == 0; }
  }
  return false;
}

cudaError_t dev_alloc_bytes(void** p, size_t bytes) {
  if(alloc_injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

cudaError_t host_pinned_alloc_bytes(void** p, size_t bytes) {
  if(alloc_injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

void alloc_checkpoint() {
  if(alloc_injected_failure()) { throw std::bad_alloc(); }
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" const char* dort_gpu_last_error(void) { return g_last_error.c_str(); }

extern "C" int dort_gpu_abi_version(void) try { return DORT_GPU_ABI_VERSION; } DORT_ABI_CATCH

extern "C" int dort_gpu_debug_fail_alloc(long long after) try {
  clear_error();
  g_alloc_budget.store(after < 0 ? -1 : after);
  return DORT_OK;
} DORT_ABI_CATCH

static void scene_free_device(dort_scene* s) {
  if(s->wavefront) { wavefront_destroy(s->wavefront); s->wavefront = nullptr; }
  if(s->adj_wavefront) { wavefront_destroy(s->adj_wavefront); s->adj_wavefront = nullptr; }
  for(void* p : s->allocations) { cudaFree(p); }
  s->allocations.clear();
  if(s->d_stage) { cudaFree(s->d_stage); }
  s->d_stage = nullptr;
  s->stage_bytes = 0;
  if(s->d_image) { cudaFree(s->d_image); }
  s->d_image = nullptr;
  s->image_bytes = 0;
  if(s->d_adjoint) { cudaFree(s->d_adjoint); }
  s->d_adjoint = nullptr;
  s->adjoint_bytes = 0;
  s->d_work = nullptr;
}

// Copies a host vector into a new device buffer owned by the scene.
template<class T>
static int upload(dort_scene* s, const std::vector<T>& v, const T** out) {
  *out = nullptr;
  if(v.empty()) { return DORT_OK; }
  void* d = nullptr;
  size_t bytes = v.size() * sizeof(T);
  if(dev_alloc(&d, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(DORT_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
  }
  s->allocations.push_back(d);
  s->device_bytes += bytes;
  DG_CUDA(cudaMemcpy(d, v.data(), bytes, cudaMemcpyHostToDevice));
  *out = static_cast<const T*>(d);
  return DORT_OK;
}

// Builds the BVH on the device (the scene owns the result).
static int device_bvh(dort_scene* s, const dort_scene_desc* desc) {
  BuildOptions opts;
  opts.width = desc->bvh_width ? desc->bvh_width : 8;
  DeviceBvh db;
  std::string err;
  DeviceBuilder method =
      desc->bvh_build == DORT_BVH_BUILD_PLOC ? DeviceBuilder::kPloc : DeviceBuilder::kSah;
  if(!build_wide_bvh_device(desc->verts, desc->vert_count, desc->tris, desc->tri_count, opts,
                            method, nullptr, db, err)) {
    int code = DORT_ERR_CUDA;
    if(err.rfind("cudaMalloc", 0) == 0 || err.find("out of memory") != std::string::npos) {
      code = DORT_ERR_OOM;
    }
    if(err.find("quantization") != std::string::npos || err.find("too ") != std::string::npos) {
      code = DORT_ERR_INVALID;
    }
    return fail(code, err);
  }
  if(db.nodes) {
    s->allocations.push_back(db.nodes);
    s->device_bytes += db.node_bytes;
  }
  if(db.tris) {
    s->allocations.push_back(db.tris);
    s->device_bytes += size_t(db.tri_count) * sizeof(LeafTri);
  }
  s->trace.nodes = static_cast<const uint4*>(db.nodes);
  s->trace.tris = reinterpret_cast<const float4*>(db.tris);
  s->trace.node_count = db.node_count;
  s->trace.tri_count = db.tri_count;
  s->depth = db.depth;
  s->bvh_ms = db.ms;
  s->bvh_builder = method == DeviceBuilder::kPloc ? DORT_BVH_BUILD_PLOC : DORT_BVH_BUILD_DEVICE;
  s->bvh_iterations = db.iterations;
  return DORT_OK;
}

// Watertight scenes: each leaf triangle's (p0, e1, e2) becomes its three
// input vertices (p0, p1, p2), taken from the shading records (by original
// triangle index), so that triangles sharing an edge hold identical
// coordinates for it.
__global__ void leaf_tris_to_vertices(float4* tris, uint32_t count, const float4* shade) {
  for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float4 a = tris[3 * size_t(i)];
    uint32_t id = __float_as_uint(a.w);
    float4 p0 = shade[3 * size_t(id)], p1 = shade[3 * size_t(id) + 1];
    float4 p2 = shade[3 * size_t(id) + 2];
    tris[3 * size_t(i)] = make_float4(p0.x, p0.y, p0.z, a.w);
    tris[3 * size_t(i) + 1] = make_float4(p1.x, p1.y, p1.z, 0.f);
    tris[3 * size_t(i) + 2] = make_float4(p2.x, p2.y, p2.z, 0.f);
  }
}

static int scene_upload(dort_scene* s, const dort_scene_desc* desc, const HostScene& hs) {
  int rc;
  if(hs.device_bvh) {
    if((rc = device_bvh(s, desc)) != DORT_OK) { return rc; }
  } else {
    const unsigned char* nodes;
    const LeafTri* tris;
    const unsigned char* src = static_cast<const unsigned char*>(traversal_nodes(hs.bvh));
    std::vector<unsigned char> bytes(src, src + traversal_node_bytes(hs.bvh));
    if((rc = upload(s, bytes, &nodes)) != DORT_OK) { return rc; }
    if((rc = upload(s, hs.bvh.tris, &tris)) != DORT_OK) { return rc; }
    s->trace.nodes = reinterpret_cast<const uint4*>(nodes);
    s->trace.tris = reinterpret_cast<const float4*>(tris);
    s->trace.node_count = uint32_t(hs.bvh.nodes.size());
    s->trace.tri_count = uint32_t(hs.bvh.tris.size());
    s->depth = hs.bvh.depth;
    s->bvh_ms = hs.bvh_ms;
    s->bvh_builder = DORT_BVH_BUILD_HOST;
  }

  PtScene& pt = s->pt;
  std::memset(&pt, 0, sizeof(pt));
  if((rc = upload(s, hs.shade, &pt.shade)) != DORT_OK) { return rc; }
  if(desc->flags & DORT_SCENE_WATERTIGHT) {
    if(s->trace.tri_count) {
      leaf_tris_to_vertices<<<std::min<uint32_t>((s->trace.tri_count + 255) / 256, 4096), 256>>>(
          const_cast<float4*>(s->trace.tris), s->trace.tri_count, pt.shade);
      DG_CUDA(cudaGetLastError());
      DG_CUDA(cudaDeviceSynchronize());
    }
    s->trace.watertight = 1;
  }
  pt.trace = s->trace;
  if((rc = upload(s, hs.mats, &pt.mats)) != DORT_OK) { return rc; }
  pt.mat_count = uint32_t(hs.mats.size());
  if((rc = upload(s, hs.lights, &pt.lights)) != DORT_OK) { return rc; }
  pt.light_count = uint32_t(hs.lights.size());
  if((rc = upload(s, hs.light_cdf, &pt.light_cdf)) != DORT_OK) { return rc; }
  pt.bg_count = hs.bg_count;
  pt.bg_light[0] = hs.bg_light[0];
  pt.bg_light[1] = hs.bg_light[1];
  pt.env = hs.env;
  if((rc = upload(s, hs.env_rgb, &pt.env.rgb)) != DORT_OK) { return rc; }
  if((rc = upload(s, hs.env_pdfs, &pt.env.pdfs)) != DORT_OK) { return rc; }
  if((rc = upload(s, hs.env_row_alias, &pt.env.row_alias)) != DORT_OK) { return rc; }
  if((rc = upload(s, hs.env_col_alias, &pt.env.col_alias)) != DORT_OK) { return rc; }
  if((rc = upload(s, hs.shapes, &pt.shapes)) != DORT_OK) { return rc; }
  pt.shape_count = uint32_t(hs.shapes.size());
  pt.shape_base = hs.shape_base;
  if((rc = upload(s, hs.light_shapes, &pt.light_shapes)) != DORT_OK) { return rc; }
  pt.general = hs.general;
  for(int a = 0; a < 3; ++a) { pt.centroid[a] = hs.centroid[a]; }
  pt.radius = hs.radius;

  void* w = nullptr;
  if(dev_alloc(&w, 64 * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return fail(DORT_ERR_OOM, "cudaMalloc of work counters failed");
  }
  s->allocations.push_back(w);
  s->device_bytes += 64 * sizeof(uint32_t);
  s->d_work = static_cast<uint32_t*>(w);
  return DORT_OK;
}

extern "C" int dort_gpu_scene_create(const dort_scene_desc* desc, dort_scene** out_scene) try {
  clear_error();
  if(!desc || !out_scene) { return fail(DORT_ERR_INVALID, "null argument"); }
  *out_scene = nullptr;

  auto t0 = std::chrono::steady_clock::now();
  HostScene hs;
  std::string err;
  if(!build_host_scene(desc, hs, err, true)) { return fail(DORT_ERR_INVALID, err); }

  dort_scene* s = new dort_scene();
  cudaGetDevice(&s->device);
  s->tri_count = desc->tri_count;
  s->emissive_count = hs.emissive_count;
  int rc;
  try {
    rc = scene_upload(s, desc, hs);
  } catch(...) {
    scene_free_device(s);
    delete s;
    throw;
  }
  s->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                    .count();
  if(rc != DORT_OK) {
    std::string msg = g_last_error;
    scene_free_device(s);
    delete s;
    return fail(rc, msg);
  }
  *out_scene = s;
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_scene_destroy(dort_scene* scene) try {
  clear_error();
  if(!scene) { return DORT_OK; }
  scene_free_device(scene);
  delete scene;
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_scene_stats(const dort_scene* s, double out[8]) try {
  clear_error();
  if(!s || !out) { return fail(DORT_ERR_INVALID, "null argument"); }
  out[0] = s->trace.node_count;
  out[1] = s->depth;
  out[2] = s->tri_count;
  out[3] = s->emissive_count;
  out[4] = double(s->device_bytes);
  out[5] = s->build_ms;
  out[6] = s->bvh_builder;
  out[7] = s->bvh_ms;
  return DORT_OK;
} DORT_ABI_CATCH
