// Autotuner of the wavefront renderer: picks the path-slot capacity and the
// thread-block sizes of the trace and shade stages for one frame (or one
// batch) by timing candidates on the GPU with CUDA events.
//
//   stage 1, block sizes: every (trace, shade) pair of {64, 128, 256} on a
//            proxy frame -- the frame's resolution, depth, camera and seed at
//            a few samples per pixel -- at 2^22 path slots;
//   stage 2, capacity:    2^22 .. 2^28 slots with the chosen
//            blocks on the frame itself (all its samples: how many waves a
//            frame takes, and so what a slot count costs, depends on the
//            whole frame's work), skipping capacities beyond twice the
//            frame's work units or beyond the device memory left (about
//            340 bytes per slot).
// Each candidate runs twice and keeps the faster run (the first builds the
// frame's graph and allocates its queues).  A time budget bounds the search;
// when it runs out the best candidate so far wins.  Batches are tuned the
// same way on a proxy batch (every job at an eighth of its spp, at least 4).
//
// No reference counterpart: the reference renders on the CPU with a fixed
// tile size.
#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "autotune_plan.h"
#include "common.h"
#include "wavefront.h"

namespace dort_gpu {
namespace {

using Clock = std::chrono::steady_clock;

constexpr uint32_t kBlocks[3] = {64, 128, 256};
constexpr uint32_t kCapacities[7] = {1u << 22, 1u << 23, 1u << 24, 1u << 25, 1u << 26,
                                      1u << 27, 1u << 28};

double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

dort_wavefront_tuning make_tuning(uint32_t cap, uint32_t tb, uint32_t sb) {
  dort_wavefront_tuning t{};
  t.struct_size = sizeof(t);
  t.queue_capacity = cap;
  t.trace_block = tb;
  t.shade_block = sb;
  return t;
}

// Milliseconds of one wavefront frame on the device (events on a private
// stream), the faster of two runs; negative status on failure.
int time_frame(dort_scene* sc, const dort_render_params* p, const dort_wavefront_tuning& t,
               float* d_out, cudaStream_t st, double* out_ms) {
  cudaEvent_t e0, e1;
  DG_CUDA(cudaEventCreate(&e0));
  DG_CUDA(cudaEventCreate(&e1));
  double best = 1e300;
  int rc = DORT_OK;
  for(int r = 0; r < 2 && rc == DORT_OK; ++r) {
    cudaEventRecord(e0, st);
    rc = dort_gpu_render_wavefront_device(sc, p, &t, d_out, st);
    cudaEventRecord(e1, st);
    if(rc == DORT_OK && cudaEventSynchronize(e1) != cudaSuccess) {
      rc = fail(DORT_ERR_CUDA, "autotune frame failed");
    }
    float ms = 0.f;
    if(rc == DORT_OK) {
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, double(ms));
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out_ms = best;
  return rc;
}

uint64_t frame_units(const dort_render_params& p) {
  // the wavefront's work units: kWfUnitSamples samples of one pixel
  return uint64_t(p.width) * p.height *
         ((p.iterations + kWfUnitSamples - 1) / kWfUnitSamples);
}

// Lights a path vertex samples (the direct-lighting queues' multiplier).
uint32_t nee_lights(const PtScene& sc, const dort_render_params& p) {
  return p.sample_all_lights ? std::max(1u, sc.light_count) : 1u;
}

}  // namespace
}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_autotune_wavefront(dort_scene* scene, const dort_render_params* params,
                                           double budget_ms, dort_wavefront_tuning* out_tuning,
                                           double* out_stats) try {
  clear_error();
  if(!scene || !params || !out_tuning) { return fail(DORT_ERR_INVALID, "null argument"); }
  if(params->struct_size != sizeof(dort_render_params) || params->renderer != DORT_RENDERER_PT) {
    return fail(DORT_ERR_INVALID, "the autotuner tunes pt frames (dort_render_params)");
  }
  if(budget_ms <= 0.0) { budget_ms = 30000.0; }
  const auto t0 = Clock::now();
  size_t npix = size_t(params->width) * params->height;
  float* d_out = nullptr;
  if(dev_alloc(&d_out, npix * 3 * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return fail(DORT_ERR_OOM, "cudaMalloc of the autotuner's image failed");
  }
  cudaStream_t st = nullptr;
  if(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(d_out);
    return fail(DORT_ERR_CUDA, "cudaStreamCreate failed");
  }
  int rc = DORT_OK;
  uint32_t timed = 0;
  bool cut = false;
  // stage 1: block sizes on a proxy frame
  dort_render_params proxy = *params;
  proxy.iterations = std::min<uint32_t>(params->iterations, 8);
  const uint32_t cap1 = uint32_t(std::min<uint64_t>(uint64_t(1) << 22,
                                                    std::max<uint64_t>(32, frame_units(proxy))));
  dort_wavefront_tuning best = make_tuning(cap1, 128, 128);
  double best_ms = 1e300;
  for(uint32_t tb : kBlocks) {
    for(uint32_t sb : kBlocks) {
      if(rc != DORT_OK) { break; }
      if(timed > 0 && ms_since(t0) > 0.3 * budget_ms) { cut = true; break; }
      dort_wavefront_tuning t = make_tuning(cap1, tb, sb);
      double ms = 0.0;
      rc = time_frame(scene, &proxy, t, d_out, st, &ms);
      ++timed;
      if(rc == DORT_OK && ms < best_ms) { best_ms = ms; best = t; }
    }
  }
  // stage 2: capacities on the frame
  const uint64_t units = frame_units(*params);
  const uint32_t nee = nee_lights(scene->pt, *params);
  uint32_t held = cap1;   // the slot count the scene's queues hold now
  double best2 = 1e300;
  dort_wavefront_tuning best_cap = best;
  best_cap.queue_capacity =
      uint32_t(std::min<uint64_t>(uint64_t(1) << 22, std::max<uint64_t>(32, units)));
  for(uint32_t cap : kCapacities) {
    if(rc != DORT_OK) { break; }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if(!capacity_candidate(cap, cap == kCapacities[0], units, nee, free_b, held)) { continue; }
    if(best2 < 1e300 && ms_since(t0) + 2.0 * best2 > budget_ms) { cut = true; break; }
    dort_wavefront_tuning t = best;
    t.queue_capacity = uint32_t(std::min<uint64_t>(cap, std::max<uint64_t>(32, units)));
    double ms = 0.0;
    const int r = time_frame(scene, params, t, d_out, st, &ms);
    ++timed;
    if(r == DORT_OK) {
      held = t.queue_capacity;
      if(ms < best2) { best2 = ms; best_cap = t; }
    } else if(r == DORT_ERR_OOM && best2 < 1e300) {
      // a larger capacity than the device holds after all: keep the best of
      // the smaller ones (the scene's queues were released by the failure)
      clear_error();
      break;
    } else {
      rc = r;
    }
  }
  cudaStreamDestroy(st);
  cudaFree(d_out);
  if(rc != DORT_OK) { return rc; }
  *out_tuning = best_cap;
  if(out_stats) {
    out_stats[0] = double(timed);
    out_stats[1] = best2;
    out_stats[2] = ms_since(t0);
    out_stats[3] = cut ? 1.0 : 0.0;
  }
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_autotune_batch(const dort_batch_job* jobs, uint32_t job_count,
                                       double budget_ms, dort_wavefront_tuning* out_tuning,
                                       double* out_stats) try {
  clear_error();
  if(!jobs || !out_tuning || job_count == 0) { return fail(DORT_ERR_INVALID, "null argument"); }
  if(budget_ms <= 0.0) { budget_ms = 60000.0; }
  const auto t0 = Clock::now();
  // the proxy batch: every job at an eighth of its samples (at least 4)
  std::vector<dort_batch_job> proxy(jobs, jobs + job_count);
  uint64_t units = 0;
  uint32_t nee = 1;
  for(auto& j : proxy) {
    j.params.iterations = std::max<uint32_t>(std::min<uint32_t>(4, j.params.iterations),
                                             j.params.iterations / 8);
    units += frame_units(j.params);
    if(j.scene) { nee = std::max(nee, nee_lights(j.scene->pt, j.params)); }
  }
  cudaStream_t st = nullptr;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = DORT_OK;
  uint32_t timed = 0;
  bool cut = false;
  dort_wavefront_tuning best = make_tuning(1u << 22, 128, 128);
  double best_ms = 1e300;
  const uint32_t caps[4] = {1u << 21, 1u << 22, 1u << 23, 1u << 24};
  for(uint32_t cap : caps) {
    if(rc != DORT_OK) { break; }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if(cap != caps[0] && !capacity_candidate(cap, false, units, nee, free_b, 0)) { continue; }
    if(best_ms < 1e300 && ms_since(t0) + 2.0 * best_ms > budget_ms) { cut = true; break; }
    dort_wavefront_tuning t = make_tuning(cap, 128, 128);
    dort_batch* b = nullptr;
    rc = dort_gpu_batch_create(proxy.data(), job_count, &t, &b);
    double ms = 1e300;
    for(int r = 0; r < 2 && rc == DORT_OK; ++r) {
      cudaEventRecord(e0, st);
      rc = dort_gpu_batch_render(b, st);
      cudaEventRecord(e1, st);
      if(rc == DORT_OK && cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(DORT_ERR_CUDA, "autotune batch failed");
      }
      float m = 0.f;
      if(rc == DORT_OK) {
        cudaEventElapsedTime(&m, e0, e1);
        ms = std::min(ms, double(m));
      }
    }
    dort_gpu_batch_destroy(b);
    ++timed;
    if(rc == DORT_OK && ms < best_ms) { best_ms = ms; best = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if(rc != DORT_OK) { return rc; }
  *out_tuning = best;
  if(out_stats) {
    out_stats[0] = double(timed);
    out_stats[1] = best_ms;
    out_stats[2] = ms_since(t0);
    out_stats[3] = cut ? 1.0 : 0.0;
  }
  return DORT_OK;
} DORT_ABI_CATCH
