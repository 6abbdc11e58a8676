// Wavefront path tracer (wavefront.cu): host-side entry points.
#pragma once
#include <cstdint>
#include <vector>

#include "pt_scene.h"

struct dort_scene;

namespace dort_gpu {

// Samples of one pixel per work unit: a path slot takes a unit, traces its
// samples one after another and adds their sum to the film once (the
// wavefront, the autotuner's slot counts and the deterministic sums' memory
// all count in units).
#ifndef DORT_WF_CHUNK
#define DORT_WF_CHUNK 1
#endif
constexpr uint32_t kWfUnitSamples = DORT_WF_CHUNK;

struct WfTuning {
  uint32_t capacity;      // paths in flight
  uint32_t trace_block;   // threads per block of extend / shadow / neeb
  uint32_t shade_block;   // threads per block of shade
  uint32_t sort;          // 1: sort each wave's rays by direction octant and origin cell
  uint32_t max_waves;     // waves a frame may take (0: the automatic bound)
  uint32_t stage_queues;  // 1: stage the shadow queue through bulk copies (TMA)
  uint32_t deterministic; // 1: per-unit sums added in unit order (single frames)
};

struct Wavefront;
void wavefront_destroy(Wavefront* wf);
int wavefront_render(dort_scene* s, const PtParams& pp, const WfTuning& tn, float* d_out,
                     cudaStream_t st);
// ms: per-stage milliseconds (5) and waves; stage_rays: extend, shadow and
// BSDF-strategy rays of the frame.
int wavefront_stage_times(dort_scene* s, const PtParams& pp, const WfTuning& tn,
                          float* d_out, cudaStream_t st, double ms[6], double stage_rays[3]);
struct WavefrontBatch;
int wavefront_batch_create(const PtScene* scenes, const PtParams* params, uint32_t n,
                           const WfTuning& tn, WavefrontBatch** out);
void wavefront_batch_destroy(WavefrontBatch* b);
int wavefront_batch_render(WavefrontBatch* b, cudaStream_t st);
int wavefront_batch_image(WavefrontBatch* b, uint32_t job, const float** d_rgb, uint32_t* npix);
int wavefront_batch_counters(WavefrontBatch* b, uint64_t* rays, uint32_t* waves,
                             uint32_t* error, cudaStream_t st);
int wavefront_counters(dort_scene* s, uint64_t* rays, uint32_t* waves, uint32_t* error,
                       cudaStream_t st);
// The adjoint's backward pass as a wavefront frame (the scene's second
// wavefront state): gradients added into d_ga / d_ge (either may be null);
// samples whose terms overflowed the per-slot log are listed in d_overflow
// as (pixel, sample), their count in *d_overflow_n (which may exceed
// overflow_cap: the list then holds the first overflow_cap).
int wavefront_adjoint(dort_scene* s, const PtParams& pp, const WfTuning& tn, const float* d_dl,
                      float* d_ga, float* d_ge, uint2* d_overflow, uint32_t overflow_cap,
                      uint32_t* d_overflow_n, cudaStream_t st);
int wavefront_adjoint_counters(dort_scene* s, uint64_t* rays, uint32_t* waves, uint32_t* error,
                               cudaStream_t st);

}  // namespace dort_gpu
