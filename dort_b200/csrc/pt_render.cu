// The plain per-pixel path tracer ("megakernel"): one thread runs whole
// paths for one pixel over a slice of its samples, keeps the sums in
// registers and writes one (sum RGB, kept count) record per (slice, pixel);
// a resolve kernel adds the slices in a fixed order and divides, so the image
// is deterministic and needs no atomics.
//
// Replaces PathRenderer::render (path_renderer.cpp:11-21) and the tiling of
// Renderer::iteration_tiled (renderer.cpp:26-86); each path is pt_sample
// (pt.cuh).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bdpt.cuh"
#include "common.h"
#include "launch_plan.h"
#include "lt.cuh"
#include "pt.cuh"
#include "scene_build.h"

namespace dort_gpu {

constexpr int kPtBlock = 128;

// Film position of sample `s` of pixel (x, y): the pixel centre on
// iteration 0, uniform jitter afterwards (path_renderer.cpp:17).
DG_HD void film_pos(const PtParams& pp, uint32_t pixel, uint32_t x, uint32_t y, uint32_t s,
                    float& fx, float& fy) {
  if(s == 0) {
    fx = float(x) + 0.5f;
    fy = float(y) + 0.5f;
  } else {
    Rand4 j = rand4(pp.seed, pixel, s, kBlockCamera);
    fx = float(x) + j.a;
    fy = float(y) + j.b;
  }
}

DG_HD bool keep_sample(V3 L) {
  // renderer.cpp:36-41: only finite, non-negative samples reach the film
  return isfinite(L.x) && isfinite(L.y) && isfinite(L.z) && L.x >= 0.f && L.y >= 0.f &&
         L.z >= 0.f;
}

// Resident blocks per SM the register allocation must allow: 5 (96
// registers) against the block size alone (168 registers): the Cornell
// workload 557 against 468 M samples/s, the 1080p frame 286.6 against 282.1
// M (6 blocks: 573 and 273.4 M).
#ifndef DORT_PT_MIN_BLOCKS
#define DORT_PT_MIN_BLOCKS 5
#endif
// 0: the block size alone (the compiler picks the registers)
#if DORT_PT_MIN_BLOCKS > 0
#define DORT_PT_BOUNDS __launch_bounds__(kPtBlock, DORT_PT_MIN_BLOCKS)
#else
#define DORT_PT_BOUNDS __launch_bounds__(kPtBlock)
#endif

template<bool G>
__global__ void DORT_PT_BOUNDS
pt_megakernel(PtScene sc, PtParams pp, uint32_t slices, uint32_t spp_per_slice,
              uint32_t per_slice, float4* __restrict__ partial,
              unsigned long long* __restrict__ ray_count) {
  const uint32_t npix = pp.width * pp.height;
  const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  uint32_t rays = 0;
  if(tid < uint64_t(per_slice) * slices) {
    // 8x4 pixel tiles per warp keep primary rays of a warp coherent; the
    // grid covers whole tiles, threads past the image edge idle
    uint32_t slice = uint32_t(tid / per_slice);
    uint32_t local = uint32_t(tid % per_slice);
    uint32_t tiles_x = (pp.width + 7) / 8;
    uint32_t tile = local / 32, lane = local % 32;
    uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
    uint32_t x = tx * 8 + lane % 8, y = ty * 4 + lane / 8;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if(x < pp.width && y < pp.height) {
      uint32_t pixel = y * pp.width + x;
      uint32_t s0 = slice * spp_per_slice;
      uint32_t s1 = min(pp.spp, s0 + spp_per_slice);
      NoTape tape;
      for(uint32_t s = s0; s < s1; ++s) {
        float fx, fy;
        film_pos(pp, pixel, x, y, s, fx, fy);
        PathResult r = pt_sample<NoTape, G>(sc, pp, pixel, s, fx, fy, tape);
        rays += r.rays;
        if(keep_sample(r.L)) {
          acc.x += r.L.x;
          acc.y += r.L.y;
          acc.z += r.L.z;
          acc.w += 1.f;
        }
      }
      partial[size_t(slice) * npix + pixel] = acc;
    }
  }
  // one atomic per warp for the ray statistics
  for(int o = 16; o > 0; o >>= 1) { rays += __shfl_down_sync(0xffffffffu, rays, o); }
  if((threadIdx.x & 31) == 0 && rays) { atomicAdd(ray_count, (unsigned long long)rays); }
}

template __global__ void pt_megakernel<false>(PtScene, PtParams, uint32_t, uint32_t, uint32_t,
                                               float4*, unsigned long long*);
template __global__ void pt_megakernel<true>(PtScene, PtParams, uint32_t, uint32_t, uint32_t,
                                              float4*, unsigned long long*);

__global__ void pt_resolve(const float4* __restrict__ partial, uint32_t slices, uint32_t npix,
                           float* __restrict__ out_rgb, unsigned long long* __restrict__ kept) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t k = 0;
  if(p < npix) {
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    for(uint32_t s = 0; s < slices; ++s) {
      float4 v = partial[size_t(s) * npix + p];
      a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
    }
    float inv = a.w != 0.f ? 1.f / a.w : 0.f;
    out_rgb[3 * size_t(p)] = a.w != 0.f ? a.x * inv : 0.f;
    out_rgb[3 * size_t(p) + 1] = a.w != 0.f ? a.y * inv : 0.f;
    out_rgb[3 * size_t(p) + 2] = a.w != 0.f ? a.z * inv : 0.f;
    k = uint32_t(a.w);
  }
  for(int o = 16; o > 0; o >>= 1) { k += __shfl_down_sync(0xffffffffu, k, o); }
  if((threadIdx.x & 31) == 0 && k) { atomicAdd(kept, (unsigned long long)k); }
}

bool make_params(const dort_render_params* rp, PtParams& pp, std::string& err) {
  if(rp->struct_size != sizeof(dort_render_params)) {
    err = "dort_render_params.struct_size mismatch (ABI version)";
    return false;
  }
  if(rp->width == 0 || rp->height == 0 || rp->width > 16384 || rp->height > 16384) {
    err = "width and height must be 1..16384";
    return false;
  }
  if(rp->iterations == 0 || rp->iterations > (1u << 20)) {
    err = "iterations must be 1..2^20";
    return false;
  }
  if(rp->max_depth > 1000) { err = "max_depth must be <= 1000"; return false; }
  if(rp->direct_strategy > 2) { err = "direct_strategy must be 0 (mis), 1 (bsdf) or 2 (light)"; return false; }
  if(rp->renderer > DORT_RENDERER_BDPT) {
    err = "renderer must be 0 (pt), 1 (lt) or 2 (bdpt)";
    return false;
  }
  if(rp->renderer == DORT_RENDERER_BDPT && rp->max_depth > 13) {
    err = "the bdpt renderer supports max_depth <= 13";
    return false;
  }
  std::memset(&pp, 0, sizeof(pp));
  const dort_camera& c = rp->camera;
  for(int a = 0; a < 3; ++a) {
    pp.origin[a] = c.origin[a];
    pp.right[a] = c.right[a];
    pp.up[a] = c.up[a];
    pp.forward[a] = c.forward[a];
  }
  // lua_camera.cpp:63-64 clamps the pinhole's field of view to [1e-2, pi]
  float fov = c.fov;
  if(c.kind == DORT_CAMERA_PINHOLE) {
    if(!(fov >= 1e-2f)) { fov = 1e-2f; }
    if(fov > kPi) { fov = kPi; }
  } else if(c.kind == DORT_CAMERA_THIN_LENS) {
    if(!(fov > 0.f && fov < kPi)) { err = "thin lens fov must be in (0, pi)"; return false; }
    if(!(c.lens_radius >= 0.f) || !std::isfinite(c.lens_radius) ||
       !(c.focal_distance > 0.f) || !std::isfinite(c.focal_distance)) {
      err = "thin lens needs lens_radius >= 0 and focal_distance > 0";
      return false;
    }
  } else if(c.kind == DORT_CAMERA_ORTHO) {
    if(!(c.dimension > 0.f) || !std::isfinite(c.dimension)) {
      err = "orthographic camera needs dimension > 0";
      return false;
    }
  } else {
    err = "unknown camera kind " + std::to_string(c.kind);
    return false;
  }
  pp.camera = c.kind;
  pp.proj_dim = 2.f * tanf(0.5f * fov);
  pp.lens_radius = c.lens_radius;
  pp.focal_distance = c.focal_distance;
  pp.ortho_dim = c.dimension;
  pp.width = rp->width;
  pp.height = rp->height;
  pp.spp = rp->iterations;
  pp.min_depth = rp->min_depth;
  pp.max_depth = rp->max_depth;
  pp.only_direct = rp->only_direct;
  pp.sample_all_lights = rp->sample_all_lights;
  pp.strategy = rp->direct_strategy;
  pp.seed = rp->seed;
  pp.renderer = rp->renderer;
  pp.use_t1 = (rp->renderer_flags & DORT_BDPT_NO_T1_PATHS) ? 0u : 1u;
  pp.roulette = (rp->renderer_flags & DORT_PT_NO_ROULETTE) ? 0u : 1u;
  if(rp->renderer_flags &
     ~(DORT_BDPT_NO_T1_PATHS | DORT_PT_NO_ROULETTE | DORT_ADJOINT_MEGAKERNEL)) {
    err = "unknown renderer_flags bits";
    return false;
  }
  // world -> camera: the inverse of the camera's linear part [right up forward]
  double m[3][3];
  for(int a = 0; a < 3; ++a) {
    m[a][0] = c.right[a];
    m[a][1] = c.up[a];
    m[a][2] = c.forward[a];
  }
  double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
               m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if(std::fabs(det) > 1e-30) {
    double inv[3][3] = {
        {m[1][1] * m[2][2] - m[1][2] * m[2][1], m[0][2] * m[2][1] - m[0][1] * m[2][2],
         m[0][1] * m[1][2] - m[0][2] * m[1][1]},
        {m[1][2] * m[2][0] - m[1][0] * m[2][2], m[0][0] * m[2][2] - m[0][2] * m[2][0],
         m[0][2] * m[1][0] - m[0][0] * m[1][2]},
        {m[1][0] * m[2][1] - m[1][1] * m[2][0], m[0][1] * m[2][0] - m[0][0] * m[2][1],
         m[0][0] * m[1][1] - m[0][1] * m[1][0]}};
    for(int r = 0; r < 3; ++r) {
      for(int k = 0; k < 3; ++k) { pp.cam_inv[3 * r + k] = float(inv[r][k] / det); }
    }
  } else if(pp.renderer != RENDERER_PT) {
    err = "the light and bidirectional tracers need an invertible camera transform";
    return false;
  }
  if(pp.renderer != RENDERER_PT && pp.camera == CAMERA_THIN_LENS && !(pp.lens_radius > 0.f)) {
    err = "the light and bidirectional tracers need a thin lens with lens_radius > 0";
    return false;
  }
  return true;
}

// Scratch for the megakernel (per-(slice, pixel) partial sums) and the light
// tracer (its film), grown on demand and kept with the scene.
int render_scratch(dort_scene* s, size_t bytes, void** out) {
  if(s->stage_bytes < bytes) {
    if(s->d_stage) { cudaFree(s->d_stage); s->d_stage = nullptr; s->stage_bytes = 0; }
    if(dev_alloc(&s->d_stage, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(DORT_ERR_OOM, "cudaMalloc of render scratch failed");
    }
    s->stage_bytes = bytes;
  }
  *out = s->d_stage;
  return DORT_OK;
}

int render_image_buffer(dort_scene* s, size_t bytes, float** out) {
  if(s->image_bytes < bytes) {
    if(s->d_image) { cudaFree(s->d_image); s->d_image = nullptr; s->image_bytes = 0; }
    if(dev_alloc(&s->d_image, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(DORT_ERR_OOM, "cudaMalloc of the image failed");
    }
    s->image_bytes = bytes;
  }
  *out = static_cast<float*>(s->d_image);
  return DORT_OK;
}

int launch_render(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                  unsigned long long* d_counters) {
  int drc = require_scene_device(s);
  if(drc != DORT_OK) { return drc; }
  if(pp.renderer == RENDERER_LT) { return launch_light_trace(s, pp, d_out, st, d_counters); }
  if(pp.renderer == RENDERER_BDPT) { return launch_bdpt(s, pp, d_out, st, d_counters); }
  int dev = 0, sms = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  uint32_t npix = pp.width * pp.height;
  // enough (pixel, slice) threads for ~4 waves of 1024 threads per SM; the
  // thread grid covers whole 8x4 pixel tiles
  MegaPlan plan;
  if(megakernel_plan(s->device, dev, sms, pp.width, pp.height, pp.spp, 0, &plan) != 0) {
    return fail(DORT_ERR_INVALID, plan.why);
  }
  const uint32_t slices = plan.slices, per = plan.per, per_slice = plan.per_slice;
  size_t partial_bytes = size_t(slices) * npix * sizeof(float4);
  void* scratch = nullptr;
  int rc = render_scratch(s, partial_bytes, &scratch);
  if(rc != DORT_OK) { return rc; }
  float4* partial = static_cast<float4*>(scratch);
  uint64_t threads = uint64_t(slices) * per_slice;
  uint32_t blocks = uint32_t((threads + kPtBlock - 1) / kPtBlock);
  if(scene_needs_general(s->pt, pp)) {
    pt_megakernel<true><<<blocks, kPtBlock, 0, st>>>(s->pt, pp, slices, per, per_slice, partial,
                                                     d_counters);
  } else {
    pt_megakernel<false><<<blocks, kPtBlock, 0, st>>>(s->pt, pp, slices, per, per_slice, partial,
                                                      d_counters);
  }
  DG_CUDA(cudaGetLastError());
  pt_resolve<<<(npix + 255) / 256, 256, 0, st>>>(partial, slices, npix, d_out, d_counters + 1);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_render_device(dort_scene* scene, const dort_render_params* params,
                                      float* d_out_rgb, void* stream) try {
  clear_error();
  if(!scene || !params || !d_out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DG_CUDA(cudaMemsetAsync(scene->d_work, 0, 2 * sizeof(unsigned long long), st));
  return launch_render(scene, pp, d_out_rgb, st,
                       reinterpret_cast<unsigned long long*>(scene->d_work));
} DORT_ABI_CATCH

extern "C" int dort_gpu_render(dort_scene* scene, const dort_render_params* params,
                               float* out_rgb, double* out_stats) try {
  clear_error();
  if(!scene || !params || !out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  size_t npix = size_t(pp.width) * pp.height;
  float* d_out = nullptr;
  int brc = render_image_buffer(scene, npix * 3 * sizeof(float), &d_out);
  if(brc != DORT_OK) { return brc; }
  cudaStream_t st = 0;
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(scene->d_work);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = DORT_OK;
  if(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st) != cudaSuccess) {
    rc = fail(DORT_ERR_CUDA, "cudaMemsetAsync failed");
  }
  if(rc == DORT_OK) {
    cudaEventRecord(e0, st);
    rc = launch_render(scene, pp, d_out, st, ctr);
    cudaEventRecord(e1, st);
  }
  unsigned long long counters[2] = {0, 0};
  if(rc == DORT_OK) {
    if(cudaMemcpyAsync(out_rgb, d_out, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaMemcpyAsync(counters, ctr, sizeof(counters), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess) {
      rc = fail(DORT_ERR_CUDA, std::string("render failed: ") + cudaGetErrorString(cudaGetLastError()));
    }
  }
  float ms = 0.f;
  if(rc == DORT_OK) { cudaEventElapsedTime(&ms, e0, e1); }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if(rc == DORT_OK && out_stats) {
    out_stats[0] = double(counters[0]);
    out_stats[1] = double(counters[1]);
    out_stats[2] = ms;
    out_stats[3] = double(uint64_t(npix) * pp.spp - counters[1]);
  }
  return rc;
} DORT_ABI_CATCH

extern "C" int dort_gpu_host_check_render(const dort_scene_desc* desc,
                                          const dort_render_params* params,
                                          uint32_t row_begin, uint32_t row_end,
                                          float* out_rgb) try {
  clear_error();
  if(!desc || !params || !out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  HostScene hs;
  std::string err;
  if(!build_host_scene(desc, hs, err)) { return fail(DORT_ERR_INVALID, err); }
  PtParams pp;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(row_end > pp.height) { row_end = pp.height; }
  PtScene sc = host_view(hs);
  if(pp.renderer != RENDERER_PT && (row_begin != 0 || row_end != pp.height)) {
    // light paths and t = 1 connections splat anywhere: whole frames only
    return fail(DORT_ERR_INVALID, "the light and bidirectional tracers' host check renders "
                                  "whole frames only");
  }
  if(pp.renderer == RENDERER_BDPT) {
    size_t npix = size_t(pp.width) * pp.height;
    std::vector<float> splat(npix * 3, 0.f);
    std::vector<double> acc(npix * 4, 0.0);
    uint32_t rays = 0;
    for(uint32_t s = 0; s < pp.spp; ++s) {
      for(uint32_t pixel = 0; pixel < npix; ++pixel) {
        Rand4 r0 = rand4(pp.seed, pixel, s, 0);
        V3 L = bdpt_sample<true>(sc, pp, pixel, s, float(pixel % pp.width) + r0.a,
                                 float(pixel / pp.width) + r0.b, pp.use_t1 != 0, splat.data(),
                                 rays);
        if(keep_sample(L)) {
          acc[4 * pixel] += L.x; acc[4 * pixel + 1] += L.y; acc[4 * pixel + 2] += L.z;
          acc[4 * pixel + 3] += 1;
        }
      }
    }
    for(size_t p = 0; p < npix; ++p) {
      double w = acc[4 * p + 3];
      for(int a = 0; a < 3; ++a) {
        out_rgb[3 * p + a] = float((w != 0 ? acc[4 * p + a] / w : 0.0) +
                                   double(splat[3 * p + a]) / pp.spp);
      }
    }
    return DORT_OK;
  }
  if(pp.renderer == RENDERER_LT) {
    size_t npix = size_t(pp.width) * pp.height;
    std::vector<float> film(npix * 3, 0.f);
    for(uint64_t i = 0; i < uint64_t(npix) * pp.spp; ++i) {
      lt_path<true>(sc, pp, uint32_t(i % npix), uint32_t(i / npix), film.data());
    }
    for(size_t k = 0; k < film.size(); ++k) { out_rgb[k] = film[k] / float(pp.spp); }
    return DORT_OK;
  }
  NoTape tape;
  for(uint32_t y = row_begin; y < row_end; ++y) {
    for(uint32_t x = 0; x < pp.width; ++x) {
      uint32_t pixel = y * pp.width + x;
      double acc[3] = {0, 0, 0};
      double w = 0;
      for(uint32_t s = 0; s < pp.spp; ++s) {
        float fx, fy;
        film_pos(pp, pixel, x, y, s, fx, fy);
        PathResult r = pt_sample<NoTape, true>(sc, pp, pixel, s, fx, fy, tape);
        if(keep_sample(r.L)) {
          acc[0] += r.L.x; acc[1] += r.L.y; acc[2] += r.L.z;
          w += 1;
        }
      }
      float* o = out_rgb + 3 * size_t(pixel);
      for(int a = 0; a < 3; ++a) { o[a] = w != 0 ? float(acc[a] / w) : 0.f; }
    }
  }
  return DORT_OK;
} DORT_ABI_CATCH

// ---- wavefront entry points -------------------------------------------------

#include "wavefront.h"

// A caller's tuning over the defaults (default_capacity path slots, 128
// threads per block, no ray sort, no queue staging, the automatic wave
// bound); false with err set on an invalid field.
static bool read_tuning(const dort_wavefront_tuning* t, uint32_t default_capacity, WfTuning& tn,
                        std::string& err) {
  tn.capacity = default_capacity;
  tn.trace_block = 128;
  tn.shade_block = 128;
  tn.sort = 0;
  tn.max_waves = 0;
  tn.stage_queues = 0;
  tn.deterministic = 0;
  if(t) {
    if(t->struct_size != sizeof(dort_wavefront_tuning)) {
      err = "dort_wavefront_tuning.struct_size mismatch (ABI version)";
      return false;
    }
    tn.max_waves = t->max_waves;
    if(t->stage_queues > 2) {
      err = "stage_queues must be 0 (auto), 1 (on) or 2 (off)";
      return false;
    }
    tn.stage_queues = t->stage_queues == 1 ? 1u : 0u;
    if(t->queue_capacity) { tn.capacity = t->queue_capacity; }
    if(t->trace_block) { tn.trace_block = t->trace_block; }
    if(t->shade_block) { tn.shade_block = t->shade_block; }
    if(t->sort_rays > 2) {
      err = "sort_rays must be 0 (auto), 1 (on) or 2 (off)";
      return false;
    }
    if(t->sort_rays == 1) { tn.sort = 1; }
    if(t->deterministic > 2) {
      err = "deterministic must be 0 (auto), 1 (on) or 2 (off)";
      return false;
    }
    tn.deterministic = t->deterministic == 1 ? 1u : 0u;
  }
  tn.capacity = (tn.capacity + 31u) & ~31u;
  if(tn.capacity < 32 || tn.capacity > (1u << 28)) {
    err = "queue_capacity must be 32..2^28";
    return false;
  }
  for(uint32_t b : {tn.trace_block, tn.shade_block}) {
    if(b < 32 || b > 1024 || b % 32 != 0) {
      err = "block sizes must be multiples of 32 in 32..1024";
      return false;
    }
  }
  return true;
}

static bool make_tuning(const dort_wavefront_tuning* t, const PtParams& pp, WfTuning& tn,
                        std::string& err) {
  uint64_t tiles = uint64_t((pp.width + 7) / 8) * ((pp.height + 3) / 4);
  uint64_t total = tiles * 32 * ((pp.spp + kWfUnitSamples - 1) / kWfUnitSamples);
  // default: up to 2^24 path slots (about 5.5 GB of path state) or the
  // frame's work units; more slots make fewer, fuller waves (the 1080p frame
  // at 256 spp: 567 M samples/s at 2^22, 606 M at 2^24 with 4-sample units;
  // the autotuner goes up to 2^28)
  return read_tuning(t, uint32_t(std::min<uint64_t>(total, 1u << 24)), tn, err);
}

extern "C" int dort_gpu_render_wavefront_device(dort_scene* scene,
                                                const dort_render_params* params,
                                                const dort_wavefront_tuning* tuning,
                                                float* d_out_rgb, void* stream) try {
  clear_error();
  if(!scene || !params || !d_out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(pp.renderer != RENDERER_PT) {
    return fail(DORT_ERR_UNSUPPORTED, "dort_gpu_render_wavefront_device renders only the pt renderer");
  }
  WfTuning tn;
  if(!make_tuning(tuning, pp, tn, err)) { return fail(DORT_ERR_INVALID, err); }
  int drc = require_scene_device(scene);
  if(drc != DORT_OK) { return drc; }
  return wavefront_render(scene, pp, tn, d_out_rgb, static_cast<cudaStream_t>(stream));
} DORT_ABI_CATCH

extern "C" int dort_gpu_render_wavefront(dort_scene* scene, const dort_render_params* params,
                                         const dort_wavefront_tuning* tuning, float* out_rgb,
                                         double* out_stats) try {
  clear_error();
  if(!scene || !params || !out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(pp.renderer != RENDERER_PT) {
    return fail(DORT_ERR_UNSUPPORTED, "dort_gpu_render_wavefront renders only the pt renderer");
  }
  size_t npix = size_t(pp.width) * pp.height;
  float* d_out = nullptr;
  int brc = render_image_buffer(scene, npix * 3 * sizeof(float), &d_out);
  if(brc != DORT_OK) { return brc; }
  cudaStream_t st = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  int rc = dort_gpu_render_wavefront_device(scene, params, tuning, d_out, st);
  cudaEventRecord(e1, st);
  uint64_t rays = 0;
  uint32_t waves = 0, error = 0;
  if(rc == DORT_OK) {
    if(cudaMemcpyAsync(out_rgb, d_out, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess) {
      rc = fail(DORT_ERR_CUDA, std::string("wavefront render failed: ") +
                               cudaGetErrorString(cudaGetLastError()));
    }
  }
  if(rc == DORT_OK) { rc = wavefront_counters(scene, &rays, &waves, &error, st); }
  if(rc == DORT_OK && error) {
    rc = fail(DORT_ERR_TIMEOUT, error & 2u ? "a wavefront stage's bounded device wait timed out"
                                           : "wavefront frame exceeded its wave limit");
  }
  float ms = 0.f;
  if(rc == DORT_OK) { cudaEventElapsedTime(&ms, e0, e1); }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if(rc == DORT_OK && out_stats) {
    out_stats[0] = double(rays);
    out_stats[1] = 0.0;
    out_stats[2] = ms;
    out_stats[3] = double(waves);
  }
  return rc;
} DORT_ABI_CATCH

extern "C" int dort_gpu_wavefront_stage_times(dort_scene* scene, const dort_render_params* params,
                                              const dort_wavefront_tuning* tuning,
                                              double out_ms[6], double out_rays[4]) try {
  clear_error();
  if(!scene || !params || !out_ms) { return fail(DORT_ERR_INVALID, "null argument"); }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(pp.renderer != RENDERER_PT) {
    return fail(DORT_ERR_UNSUPPORTED, "dort_gpu_wavefront_stage_times renders only the pt renderer");
  }
  WfTuning tn;
  if(!make_tuning(tuning, pp, tn, err)) { return fail(DORT_ERR_INVALID, err); }
  int drc = require_scene_device(scene);
  if(drc != DORT_OK) { return drc; }
  size_t npix = size_t(pp.width) * pp.height;
  float* d_out = nullptr;
  int brc = render_image_buffer(scene, npix * 3 * sizeof(float), &d_out);
  if(brc != DORT_OK) { return brc; }
  double stage_rays[3];
  int rc = wavefront_stage_times(scene, pp, tn, d_out, 0, out_ms, stage_rays);
  if(rc == DORT_OK) {
    uint64_t rays = 0;
    uint32_t waves = 0, error = 0;
    rc = wavefront_counters(scene, &rays, &waves, &error, 0);
    out_ms[5] = double(waves);
    if(out_rays) {
      out_rays[0] = double(rays);
      for(int k = 0; k < 3; ++k) { out_rays[k + 1] = stage_rays[k]; }
    }
  }
  return rc;
} DORT_ABI_CATCH

// ---- batches ------------------------------------------------------------------

struct dort_batch {
  dort_gpu::WavefrontBatch* impl = nullptr;
  uint64_t total_samples = 0;
};

extern "C" int dort_gpu_batch_create(const dort_batch_job* jobs, uint32_t job_count,
                                     const dort_wavefront_tuning* tuning,
                                     dort_batch** out_batch) try {
  clear_error();
  if(!jobs || !out_batch || job_count == 0) { return fail(DORT_ERR_INVALID, "null argument"); }
  if(job_count > 65536) { return fail(DORT_ERR_INVALID, "job_count exceeds 65536"); }
  *out_batch = nullptr;
  std::vector<PtScene> scenes(job_count);
  std::vector<PtParams> params(job_count);
  uint64_t total = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  for(uint32_t j = 0; j < job_count; ++j) {
    if(!jobs[j].scene) { return fail(DORT_ERR_INVALID, "job " + std::to_string(j) + ": null scene"); }
    if(jobs[j].scene->device != dev) {
      return fail(DORT_ERR_INVALID, "job " + std::to_string(j) + ": scene on another device");
    }
    std::string err;
    if(!make_params(&jobs[j].params, params[j], err)) {
      return fail(DORT_ERR_INVALID, "job " + std::to_string(j) + ": " + err);
    }
    if(params[j].renderer != RENDERER_PT) {
      return fail(DORT_ERR_UNSUPPORTED, "job " + std::to_string(j) + ": batches render only pt");
    }
    scenes[j] = jobs[j].scene->pt;
    total += uint64_t(params[j].width) * params[j].height * params[j].spp;
  }
  WfTuning tn;
  std::string terr;
  // batches keep 2^22 slots: the batch workload measured 192 M samples/s at
  // 2^22 and 187 M at 2^24
  if(!read_tuning(tuning, uint32_t(std::min<uint64_t>(total, 1u << 22)), tn, terr)) {
    return fail(DORT_ERR_INVALID, terr);
  }
  if(tn.deterministic) {
    return fail(DORT_ERR_UNSUPPORTED, "deterministic sums are for single frames, not batches");
  }
  auto* batch = new dort_batch();
  int rc = wavefront_batch_create(scenes.data(), params.data(), job_count, tn, &batch->impl);
  if(rc != DORT_OK) {
    delete batch;
    return rc;
  }
  batch->total_samples = total;
  *out_batch = batch;
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_batch_render(dort_batch* batch, void* stream) try {
  clear_error();
  if(!batch) { return fail(DORT_ERR_INVALID, "null argument"); }
  return wavefront_batch_render(batch->impl, static_cast<cudaStream_t>(stream));
} DORT_ABI_CATCH

extern "C" int dort_gpu_batch_image_device(dort_batch* batch, uint32_t job,
                                           const float** out_d_rgb) try {
  clear_error();
  if(!batch || !out_d_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  uint32_t npix = 0;
  return wavefront_batch_image(batch->impl, job, out_d_rgb, &npix);
} DORT_ABI_CATCH

extern "C" int dort_gpu_batch_image(dort_batch* batch, uint32_t job, float* out_rgb) try {
  clear_error();
  if(!batch || !out_rgb) { return fail(DORT_ERR_INVALID, "null argument"); }
  const float* d = nullptr;
  uint32_t npix = 0;
  int rc = wavefront_batch_image(batch->impl, job, &d, &npix);
  if(rc != DORT_OK) { return rc; }
  DG_CUDA(cudaMemcpy(out_rgb, d, size_t(npix) * 3 * sizeof(float), cudaMemcpyDeviceToHost));
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_batch_stats(dort_batch* batch, double out[4]) try {
  clear_error();
  if(!batch || !out) { return fail(DORT_ERR_INVALID, "null argument"); }
  DG_CUDA(cudaDeviceSynchronize());
  uint64_t rays = 0;
  uint32_t waves = 0, error = 0;
  int rc = wavefront_batch_counters(batch->impl, &rays, &waves, &error, 0);
  if(rc != DORT_OK) { return rc; }
  out[0] = double(rays);
  out[1] = double(waves);
  out[2] = double(error);
  out[3] = double(batch->total_samples);
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_batch_destroy(dort_batch* batch) try {
  clear_error();
  if(!batch) { return DORT_OK; }
  wavefront_batch_destroy(batch->impl);
  delete batch;
  return DORT_OK;
} DORT_ABI_CATCH
