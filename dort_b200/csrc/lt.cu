// The "lt" renderer (LightRenderer, light_renderer.cpp:13-181) on the device:
// one persistent grid walks the frame's W x H x iterations light paths
// (lt.cuh) and splats onto a float film with atomic adds; a resolve pass
// scales the film by 1 / iterations into the caller's image.
#include <algorithm>

#include "common.h"
#include "lt.cuh"

namespace dort_gpu {

constexpr int kLtBlock = 128;
// Resident blocks per SM the register allocation must allow: 8 (64
// registers, with spills) ran the Cornell workload at 867 M samples/s
// against 817 M with the block size alone (128 registers, 4 blocks) and 712 M
// at 6; the light paths' visibility rays and splats wait on memory, which
// more resident warps hide.  (An explicit minimum of 1 is not the same as
// none: the compiler then took 180 registers.)
#ifndef DORT_LT_MIN_BLOCKS
#define DORT_LT_MIN_BLOCKS 8
#endif
// 0: the block size alone (the compiler picks the registers)
#if DORT_LT_MIN_BLOCKS > 0
#define DORT_LT_BOUNDS __launch_bounds__(kLtBlock, DORT_LT_MIN_BLOCKS)
#else
#define DORT_LT_BOUNDS __launch_bounds__(kLtBlock)
#endif

template<bool G>
__global__ void DORT_LT_BOUNDS
lt_kernel(PtScene sc, PtParams pp, uint64_t paths, float* __restrict__ film,
          unsigned long long* __restrict__ counters) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint32_t npix = pp.width * pp.height;
  unsigned long long rays = 0, done = 0;
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < paths; i += stride) {
    uint32_t pixel = uint32_t(i % npix), sample = uint32_t(i / npix);
    rays += lt_path<G>(sc, pp, pixel, sample, film);
    ++done;
  }
  for(int o = 16; o > 0; o >>= 1) {
    rays += __shfl_down_sync(0xffffffffu, rays, o);
    done += __shfl_down_sync(0xffffffffu, done, o);
  }
  if((threadIdx.x & 31) == 0 && done) {
    atomicAdd(&counters[0], rays);
    atomicAdd(&counters[1], done);
  }
}

__global__ void lt_resolve(const float* __restrict__ film, size_t count, float scale,
                           float* __restrict__ out) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if(i < count) { out[i] = film[i] * scale; }
}

int launch_light_trace(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                       unsigned long long* d_counters) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  size_t npix = size_t(pp.width) * pp.height;
  void* scratch = nullptr;
  int rc = render_scratch(s, npix * 3 * sizeof(float), &scratch);
  if(rc != DORT_OK) { return rc; }
  float* film = static_cast<float*>(scratch);
  DG_CUDA(cudaMemsetAsync(film, 0, npix * 3 * sizeof(float), st));
  uint64_t paths = uint64_t(npix) * pp.spp;
  uint64_t want = (paths + kLtBlock - 1) / kLtBlock;
  uint32_t blocks = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(sms) * 8)));
  if(scene_needs_general(s->pt, pp)) {
    lt_kernel<true><<<blocks, kLtBlock, 0, st>>>(s->pt, pp, paths, film, d_counters);
  } else {
    lt_kernel<false><<<blocks, kLtBlock, 0, st>>>(s->pt, pp, paths, film, d_counters);
  }
  DG_CUDA(cudaGetLastError());
  size_t count = npix * 3;
  lt_resolve<<<uint32_t((count + 255) / 256), 256, 0, st>>>(film, count, 1.f / float(pp.spp),
                                                            d_out);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

}  // namespace dort_gpu
