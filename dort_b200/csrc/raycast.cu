// Ray-cast kernels and their C-ABI entry points.
//
// One thread per ray inside a persistent grid (one wave of resident blocks);
// each warp takes 32 consecutive rays at a time from a device work counter,
// so warps whose rays finish early pick up new ones instead of idling until
// the slowest ray of a static block is done.  Rays are read as two 16-byte
// loads, results written as one u32 + three floats per ray.
#include <cstring>
#include <string>

#include "common.h"
#include "trace.cuh"

namespace dort_gpu {

constexpr int kRaycastBlock = 128;
// The work counter runs past ray_count by at most one fetch per warp; entries
// are limited so that it cannot wrap.
constexpr size_t kRaycastMaxRays = 0xff000000u;

// Launch bound without a minimum block count (DORT_RAYCAST_MIN_BLOCKS
// unset): the compiler then keeps the kernel at 60-64 registers, 2,476
// Mrays/s on the ray-cast workload.  An explicit minimum of 1 raised it to 96
// registers (2,044 Mrays/s); minimums of 9, 10, 12 and 16 measured 2,384,
// 2,001, 1,309 and 692 Mrays/s.
#ifdef DORT_RAYCAST_MIN_BLOCKS
#define DORT_RAYCAST_BOUNDS __launch_bounds__(kRaycastBlock, DORT_RAYCAST_MIN_BLOCKS)
#else
#define DORT_RAYCAST_BOUNDS __launch_bounds__(kRaycastBlock)
#endif
template<bool ANY_HIT, int WT = kTriMt>
__global__ void DORT_RAYCAST_BOUNDS
raycast_kernel(TraceScene sc, const float4* __restrict__ rays, uint32_t ray_count,
               uint32_t* __restrict__ out_prim, float* __restrict__ out_tb,
               uint32_t* __restrict__ work) {
  const uint32_t lane = threadIdx.x & 31u;
  for(;;) {
    uint32_t base = 0;
    if(lane == 0) { base = atomicAdd(work, 32u); }
    base = __shfl_sync(0xffffffffu, base, 0);
    if(base >= ray_count) { break; }
    uint32_t i = base + lane;
    if(i < ray_count) {
      float4 r0 = __ldcs(rays + 2 * size_t(i));
      float4 r1 = __ldcs(rays + 2 * size_t(i) + 1);
      Hit h = trace_ray<ANY_HIT, true, WT>(sc, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w);
      if(ANY_HIT) {
        out_prim[i] = h.prim != kMiss ? 1u : 0u;
      } else {
        out_prim[i] = h.prim;
        if(h.prim != kMiss) {
          out_tb[3 * size_t(i)] = h.t;
          out_tb[3 * size_t(i) + 1] = h.b1;
          out_tb[3 * size_t(i) + 2] = h.b2;
        }
      }
    }
  }
}

static int persistent_blocks(const void* kernel, int block) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
  if(per_sm < 1) { per_sm = 1; }
  return sms * per_sm;
}

int launch_raycast(dort_scene* s, const float* d_rays, size_t n, int any_hit,
                   uint32_t* d_prim, float* d_tb, cudaStream_t stream) {
  if(n == 0) { return DORT_OK; }
  if(n > kRaycastMaxRays) { return fail(DORT_ERR_INVALID, "ray_count exceeds 2^32 - 2^24"); }
  if(reinterpret_cast<uintptr_t>(d_rays) % 16 != 0) {
    return fail(DORT_ERR_INVALID, "rays must be 16-byte aligned");
  }
  if(!any_hit && !d_tb) { return fail(DORT_ERR_INVALID, "out_tb is required for closest hit"); }
  int drc = require_scene_device(s);
  if(drc != DORT_OK) { return drc; }
  DG_CUDA(cudaMemsetAsync(s->d_work, 0, sizeof(uint32_t), stream));
  const bool wt = s->trace.watertight != 0;
  const void* kfn =
      wt ? (any_hit ? reinterpret_cast<const void*>(&raycast_kernel<true, kTriWatertight>)
                    : reinterpret_cast<const void*>(&raycast_kernel<false, kTriWatertight>))
         : (any_hit ? reinterpret_cast<const void*>(&raycast_kernel<true>)
                    : reinterpret_cast<const void*>(&raycast_kernel<false>));
  static int blocks_cache[4] = {0, 0, 0, 0};
  int& blocks = blocks_cache[(wt ? 2 : 0) + (any_hit ? 1 : 0)];
  if(blocks == 0) { blocks = persistent_blocks(kfn, kRaycastBlock); }
  const float4* r4 = reinterpret_cast<const float4*>(d_rays);
  if(wt && any_hit) {
    raycast_kernel<true, kTriWatertight><<<blocks, kRaycastBlock, 0, stream>>>(
        s->trace, r4, uint32_t(n), d_prim, d_tb, s->d_work);
  } else if(wt) {
    raycast_kernel<false, kTriWatertight><<<blocks, kRaycastBlock, 0, stream>>>(
        s->trace, r4, uint32_t(n), d_prim, d_tb, s->d_work);
  } else if(any_hit) {
    raycast_kernel<true><<<blocks, kRaycastBlock, 0, stream>>>(
        s->trace, r4, uint32_t(n), d_prim, d_tb, s->d_work);
  } else {
    raycast_kernel<false><<<blocks, kRaycastBlock, 0, stream>>>(
        s->trace, r4, uint32_t(n), d_prim, d_tb, s->d_work);
  }
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_raycast_device(dort_scene* scene, const float* d_rays,
                                       size_t ray_count, int any_hit, uint32_t* d_prim,
                                       float* d_tb, void* stream) try {
  clear_error();
  if(!scene || (ray_count && (!d_rays || !d_prim))) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  return launch_raycast(scene, d_rays, ray_count, any_hit, d_prim, d_tb,
                        static_cast<cudaStream_t>(stream));
} DORT_ABI_CATCH

extern "C" int dort_gpu_raycast(dort_scene* scene, const float* rays, size_t ray_count,
                                int any_hit, uint32_t* out_prim, float* out_tb) try {
  clear_error();
  if(!scene || (ray_count && (!rays || !out_prim || (!any_hit && !out_tb)))) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  if(ray_count == 0) { return DORT_OK; }
  size_t ray_bytes = ray_count * 8 * sizeof(float);
  size_t prim_bytes = ray_count * sizeof(uint32_t);
  size_t tb_bytes = ray_count * 3 * sizeof(float);
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t need = align(ray_bytes) + align(prim_bytes) + align(tb_bytes);
  if(scene->stage_bytes < need) {
    if(scene->d_stage) { cudaFree(scene->d_stage); scene->d_stage = nullptr; }
    if(dev_alloc(&scene->d_stage, need) != cudaSuccess) {
      cudaGetLastError();
      scene->stage_bytes = 0;
      return fail(DORT_ERR_OOM, "cudaMalloc of ray staging buffer failed");
    }
    scene->stage_bytes = need;
  }
  char* base = static_cast<char*>(scene->d_stage);
  float* d_rays = reinterpret_cast<float*>(base);
  uint32_t* d_prim = reinterpret_cast<uint32_t*>(base + align(ray_bytes));
  float* d_tb = reinterpret_cast<float*>(base + align(ray_bytes) + align(prim_bytes));
  cudaStream_t st = 0;
  DG_CUDA(cudaMemcpyAsync(d_rays, rays, ray_bytes, cudaMemcpyHostToDevice, st));
  if(!any_hit) {
    // misses leave out_tb untouched: start from the caller's contents
    DG_CUDA(cudaMemcpyAsync(d_tb, out_tb, tb_bytes, cudaMemcpyHostToDevice, st));
  }
  int rc = launch_raycast(scene, d_rays, ray_count, any_hit, d_prim, d_tb, st);
  if(rc != DORT_OK) { return rc; }
  DG_CUDA(cudaMemcpyAsync(out_prim, d_prim, prim_bytes, cudaMemcpyDeviceToHost, st));
  if(!any_hit) {
    DG_CUDA(cudaMemcpyAsync(out_tb, d_tb, tb_bytes, cudaMemcpyDeviceToHost, st));
  }
  DG_CUDA(cudaStreamSynchronize(st));
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_raycast_timed(dort_scene* scene, const float* d_rays,
                                      size_t ray_count, int any_hit, uint32_t* d_prim,
                                      float* d_tb, void* stream, int repeat,
                                      float* out_ms_per_launch) try {
  clear_error();
  if(!scene || !out_ms_per_launch || repeat < 1) {
    return fail(DORT_ERR_INVALID, "bad argument");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  DG_CUDA(cudaEventCreate(&e0));
  DG_CUDA(cudaEventCreate(&e1));
  DG_CUDA(cudaEventRecord(e0, st));
  for(int r = 0; r < repeat; ++r) {
    int rc = launch_raycast(scene, d_rays, ray_count, any_hit, d_prim, d_tb, st);
    if(rc != DORT_OK) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
  }
  DG_CUDA(cudaEventRecord(e1, st));
  DG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  DG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out_ms_per_launch = ms / float(repeat);
  return DORT_OK;
} DORT_ABI_CATCH
