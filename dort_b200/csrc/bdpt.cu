// The "bdpt" renderer (BdptRenderer, bdpt_renderer.cpp:9-468) on the device:
// one thread per pixel sample (grid-stride over W x H x iterations), the
// camera-side value added to its pixel with one float4 atomic (sum, count:
// only finite, non-negative samples, renderer.cpp:36-41), t = 1 connections
// splatted onto a second film; a resolve pass adds the splats scaled by
// 1 / iterations (the film's splat_scale at the end of render, :21-31).
#include <algorithm>

#include "bdpt.cuh"
#include "common.h"

namespace dort_gpu {

constexpr int kBdptBlock = 128;
// Resident blocks per SM the register allocation must allow.
#ifndef DORT_BDPT_MIN_BLOCKS
#define DORT_BDPT_MIN_BLOCKS 1
#endif

template<bool G>
__global__ void __launch_bounds__(kBdptBlock, DORT_BDPT_MIN_BLOCKS)
bdpt_kernel(PtScene sc, PtParams pp, uint64_t total, float4* __restrict__ acc,
            float* __restrict__ splat, unsigned long long* __restrict__ counters) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint32_t npix = pp.width * pp.height;
  uint32_t rays = 0;
  unsigned long long kept = 0;
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    uint32_t pixel = uint32_t(i % npix), sample = uint32_t(i / npix);
    uint32_t x = pixel % pp.width, y = pixel / pp.width;
    Rand4 r0 = rand4(pp.seed, pixel, sample, 0);
    V3 L = bdpt_sample<G>(sc, pp, pixel, sample, float(x) + r0.a, float(y) + r0.b,
                          pp.use_t1 != 0, splat, rays);
    if(isfinite(L.x) && isfinite(L.y) && isfinite(L.z) && L.x >= 0.f && L.y >= 0.f &&
       L.z >= 0.f) {
      atomicAdd(&acc[pixel], make_float4(L.x, L.y, L.z, 1.f));
      ++kept;
    }
  }
  unsigned long long r = rays;
  for(int o = 16; o > 0; o >>= 1) {
    r += __shfl_down_sync(0xffffffffu, r, o);
    kept += __shfl_down_sync(0xffffffffu, kept, o);
  }
  if((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[0], r);
    atomicAdd(&counters[1], kept);
  }
}

__global__ void bdpt_resolve(const float4* __restrict__ acc, const float* __restrict__ splat,
                             uint32_t npix, float splat_scale, float* __restrict__ out) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if(p >= npix) { return; }
  float4 a = acc[p];
  float inv = a.w != 0.f ? 1.f / a.w : 0.f;
  out[3 * size_t(p)] = a.x * inv + splat[3 * size_t(p)] * splat_scale;
  out[3 * size_t(p) + 1] = a.y * inv + splat[3 * size_t(p) + 1] * splat_scale;
  out[3 * size_t(p) + 2] = a.z * inv + splat[3 * size_t(p) + 2] * splat_scale;
}

int launch_bdpt(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                unsigned long long* d_counters) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  size_t npix = size_t(pp.width) * pp.height;
  size_t acc_bytes = npix * sizeof(float4), splat_bytes = npix * 3 * sizeof(float);
  void* scratch = nullptr;
  int rc = render_scratch(s, acc_bytes + splat_bytes, &scratch);
  if(rc != DORT_OK) { return rc; }
  float4* acc = static_cast<float4*>(scratch);
  float* splat = reinterpret_cast<float*>(static_cast<char*>(scratch) + acc_bytes);
  DG_CUDA(cudaMemsetAsync(scratch, 0, acc_bytes + splat_bytes, st));
  uint64_t total = uint64_t(npix) * pp.spp;
  uint64_t want = (total + kBdptBlock - 1) / kBdptBlock;
  uint32_t blocks = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(sms) * 8)));
  // one instantiation: the bidirectional tracer is not specialised
  bdpt_kernel<true><<<blocks, kBdptBlock, 0, st>>>(s->pt, pp, total, acc, splat, d_counters);
  DG_CUDA(cudaGetLastError());
  bdpt_resolve<<<uint32_t((npix + 255) / 256), 256, 0, st>>>(acc, splat, uint32_t(npix),
                                                             1.f / float(pp.spp), d_out);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

}  // namespace dort_gpu
