// Adjoint of the path tracer: gradients of an image loss with respect to
// per-triangle Lambert albedo and per-triangle emitted radiance, by path
// replay backpropagation (Vicini, Speierer, Jakob, "Path Replay
// Backpropagation", SIGGRAPH 2021).  Every sample is traced from its
// counter-based random numbers with an observer that keeps the sum A of the
// terms seen so far and attributes derivatives once the sample value L is
// known:
//     - a Lambert vertex on triangle t: every later term of the sample is
//       linear in that vertex's albedo, so dL/d(albedo_t) += (L - A) / albedo_t
//       (per channel);
//     - an emission term throughput * Le of light triangle t:
//       dL/d(Le_t) += throughput;
//     - a direct-lighting term c from light triangle t: dL/d(Le_t) += c / Le_t.
// Sampling decisions (light choice, Russian roulette probabilities, MIS
// weights) are held fixed, which keeps the gradient estimate unbiased.  The
// image gradient dLoss/dI weights each sample by dLoss/dI(pixel) / spp, and
// gradients are accumulated with float atomics.
//
// One pass per sample: the observer (AdjointLog) records each term's
// triangle and factor in a short per-thread log and applies them after the
// path ends, when L is known -- a sample the film drops adds nothing.  A
// path with more terms than the log holds is traced a second time with an
// observer that applies each term as it comes (AdjointTape, given L from
// the first pass): the replay of the paper, which stores no vertex at all.
//
// No reference counterpart: the reference renderer has no derivatives.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "adjoint.cuh"
#include "common.h"
#include "launch_plan.h"
#include "pt.cuh"
#include "scene_build.h"
#include "wavefront.h"

namespace dort_gpu {

bool make_params(const dort_render_params* rp, PtParams& pp, std::string& err);
int launch_render(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                  unsigned long long* d_counters);

// The observer only runs on the device (atomics); its host instantiation of
// the shared path code is never called.
#ifdef __CUDA_ARCH__
#define ADJ_ADD(p, v) atomicAdd((p), (v))
#else
#define ADJ_ADD(p, v) (*(p) += (v))
#endif

struct AdjointTape {
  V3 L;          // sample value from pass 1
  V3 acc;        // terms seen so far
  V3 adj;        // dLoss/dI(pixel) / spp
  float* d_albedo;
  float* d_emission;
  const float* tri_emission;
  uint32_t tri_count;   // prims at or above it are analytic shapes (no gradient)

  DG_HD void emission(uint32_t tri, V3 thr, V3 Le) {
    acc = acc + thr * Le;
    if(d_emission && !is_black(Le) && tri < tri_count) {
      float* g = d_emission + 3 * size_t(tri);
      ADJ_ADD(g, adj.x * thr.x);
      ADJ_ADD(g + 1, adj.y * thr.y);
      ADJ_ADD(g + 2, adj.z * thr.z);
    }
  }
  DG_HD void background(V3 c) { acc = acc + c; }
  DG_HD void vertex(uint32_t tri, const DevMaterial& m) {
    if(!d_albedo || !adj_albedo_vertex(m, tri, tri_count)) { return; }
    V3 rem = L - acc;
    float* g = d_albedo + 3 * size_t(tri);
    if(m.c[0] > 0.f) { ADJ_ADD(g, adj.x * rem.x / m.c[0]); }
    if(m.c[1] > 0.f) { ADJ_ADD(g + 1, adj.y * rem.y / m.c[1]); }
    if(m.c[2] > 0.f) { ADJ_ADD(g + 2, adj.z * rem.z / m.c[2]); }
  }
  DG_HD void direct(uint32_t light_tri, V3 c) {
    acc = acc + c;
    if(d_emission && light_tri != kMiss) {
      const float* le = tri_emission + 3 * size_t(light_tri);
      float* g = d_emission + 3 * size_t(light_tri);
      if(le[0] > 0.f) { ADJ_ADD(g, adj.x * c.x / le[0]); }
      if(le[1] > 0.f) { ADJ_ADD(g + 1, adj.y * c.y / le[1]); }
      if(le[2] > 0.f) { ADJ_ADD(g + 2, adj.z * c.z / le[2]); }
    }
  }
};

// Terms of one sample in a per-thread log (adjoint.cuh's entries).
struct AdjointLog {
  float4 ev[kAdjLog];
  uint32_t n;
  bool overflow;
  bool want_albedo, want_emission;
  uint32_t tri_count;
  V3 acc;

  DG_HD void init(bool albedo, bool emission, uint32_t tris) {
    n = 0;
    overflow = false;
    want_albedo = albedo;
    want_emission = emission;
    tri_count = tris;
    acc = v3(0.f, 0.f, 0.f);
  }
  DG_HD void push(uint32_t kind, uint32_t prim, V3 v) {
    if(n >= kAdjLog || prim > kEvPrimMask) { overflow = true; return; }
    ev[n++] = adj_entry(kind, prim, v);
  }
  DG_HD void emission(uint32_t tri, V3 thr, V3 Le) {
    acc = acc + thr * Le;
    if(want_emission && !is_black(Le) && tri < tri_count) { push(kEvEmission, tri, thr); }
  }
  DG_HD void background(V3 c) { acc = acc + c; }
  DG_HD void vertex(uint32_t tri, const DevMaterial& m) {
    if(!want_albedo || !adj_albedo_vertex(m, tri, tri_count)) { return; }
    if(n + 2 > kAdjLog) { overflow = true; return; }
    push(kEvVertex, tri, acc);
    push(kEvVertex, tri, v3(m.c[0], m.c[1], m.c[2]));
  }
  DG_HD void direct(uint32_t light_tri, V3 c) {
    acc = acc + c;
    if(want_emission && light_tri != kMiss) { push(kEvDirect, light_tri, c); }
  }
  __device__ void apply(V3 L, V3 adj, const float* tri_emission, float* d_albedo,
                        float* d_emission) const {
    adj_apply(ev, 1, n, L, adj, tri_emission, d_albedo, d_emission);
  }
};

constexpr int kAdjBlock = 128;
// Path slots of the wavefront backward pass (one per 4-sample work unit of
// the frame, at most this many; each slot's term log takes 512 bytes).
constexpr uint64_t kAdjSlots = uint64_t(1) << 22;
// Entries of the list of samples traced a second time (8 bytes each).
constexpr uint64_t kAdjListMax = uint64_t(1) << 24;
// A smaller list for tests of the path taken when it fills (-1: none).
std::atomic<long long> g_adj_list_cap{-1};
// Resident blocks per SM the register allocation must allow: 3 caps the
// kernel at 168 registers (214 unbounded, 2 blocks), with a few bytes of
// spill; the adjoint workload (512 x 512, 64 spp, depth 6, 500k triangles)
// measured 295 ms against 339 ms per forward + backward.  4 blocks (128
// registers) spill hundreds of bytes per thread.
#ifndef DORT_ADJ_MIN_BLOCKS
#define DORT_ADJ_MIN_BLOCKS 3
#endif

// One sample's gradient: its path traced once with the term log; a path
// whose terms overflow the log is traced again with immediate attribution.
template<bool G>
__device__ __forceinline__ void adjoint_sample(const PtScene& sc, const PtParams& pp,
                                               uint32_t pixel, uint32_t s, V3 adj,
                                               float* d_albedo, float* d_emission) {
  const uint32_t x = pixel % pp.width, y = pixel / pp.width;
  float fx, fy;
  if(s == 0) {
    fx = float(x) + 0.5f;
    fy = float(y) + 0.5f;
  } else {
    Rand4 j = rand4(pp.seed, pixel, s, kBlockCamera);
    fx = float(x) + j.a;
    fy = float(y) + j.b;
  }
  AdjointLog log;
  log.init(d_albedo != nullptr, d_emission != nullptr, sc.shape_base);
  PathResult r1 = pt_sample<AdjointLog, G>(sc, pp, pixel, s, fx, fy, log);
  V3 L = r1.L;
  // samples the film drops have no gradient (renderer.cpp:36-41)
  if(!adj_kept(L)) { return; }
  if(!log.overflow) {
    log.apply(L, adj, sc.tri_emission, d_albedo, d_emission);
    return;
  }
  AdjointTape tape;
  tape.L = L;
  tape.acc = v3(0.f, 0.f, 0.f);
  tape.adj = adj;
  tape.d_albedo = d_albedo;
  tape.d_emission = d_emission;
  tape.tri_emission = sc.tri_emission;
  tape.tri_count = sc.shape_base;
  pt_sample<AdjointTape, G>(sc, pp, pixel, s, fx, fy, tape);
}

__device__ __forceinline__ V3 pixel_adj(const float* dl_dimage, uint32_t pixel, float inv_spp) {
  return v3(dl_dimage[3 * size_t(pixel)], dl_dimage[3 * size_t(pixel) + 1],
            dl_dimage[3 * size_t(pixel) + 2]) * inv_spp;
}

// The backward pass as a megakernel: one thread per (pixel, slice of samples),
// 8 x 4 pixel tiles per warp.
template<bool G>
__global__ void __launch_bounds__(kAdjBlock, DORT_ADJ_MIN_BLOCKS)
adjoint_replay(PtScene sc, PtParams pp, uint32_t slices, uint32_t spp_per_slice,
               uint32_t per_slice, const float* __restrict__ dl_dimage,
               float* __restrict__ d_albedo, float* __restrict__ d_emission) {
  const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if(tid >= uint64_t(per_slice) * slices) { return; }
  uint32_t slice = uint32_t(tid / per_slice);
  uint32_t local = uint32_t(tid % per_slice);
  uint32_t tiles_x = (pp.width + 7) / 8;
  uint32_t tile = local / 32, lane = local % 32;
  uint32_t x = (tile % tiles_x) * 8 + lane % 8, y = (tile / tiles_x) * 4 + lane / 8;
  if(x >= pp.width || y >= pp.height) { return; }
  uint32_t pixel = y * pp.width + x;
  V3 adj = pixel_adj(dl_dimage, pixel, 1.f / float(pp.spp));
  if(is_black(adj)) { return; }
  uint32_t s0 = slice * spp_per_slice;
  uint32_t s1 = min(pp.spp, s0 + spp_per_slice);
  for(uint32_t s = s0; s < s1; ++s) {
    adjoint_sample<G>(sc, pp, pixel, s, adj, d_albedo, d_emission);
  }
}

// The samples the wavefront backward could not log (list of pixel, sample).
template<bool G>
__global__ void __launch_bounds__(kAdjBlock, DORT_ADJ_MIN_BLOCKS)
adjoint_replay_list(PtScene sc, PtParams pp, const uint2* __restrict__ list, uint32_t n,
                    const float* __restrict__ dl_dimage, float* __restrict__ d_albedo,
                    float* __restrict__ d_emission) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  const uint2 e = list[i];
  V3 adj = pixel_adj(dl_dimage, e.x, 1.f / float(pp.spp));
  if(is_black(adj)) { return; }
  adjoint_sample<G>(sc, pp, e.x, e.y, adj, d_albedo, d_emission);
}

__global__ void l2_loss_grad(const float* __restrict__ img, const float* __restrict__ target,
                             uint32_t n, float* __restrict__ grad, double* __restrict__ loss) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if(i < n) {
    float d = img[i] - target[i];
    grad[i] = 2.f * d;
    l = double(d) * double(d);
  }
  for(int o = 16; o > 0; o >>= 1) { l += __shfl_down_sync(0xffffffffu, l, o); }
  if((threadIdx.x & 31) == 0 && l != 0.0) { atomicAdd(loss, l); }
}

// Per-triangle parameter overrides held by the scene: one device buffer each,
// allocated on first use and overwritten by later calls; NULL clears.
static int set_tri_params(dort_scene* s, const float* albedo, const float* emission) {
  size_t n = size_t(s->tri_count) * 3;
  size_t bytes = n * sizeof(float);
  for(size_t i = 0; albedo && i < n; ++i) {
    if(!std::isfinite(albedo[i]) || albedo[i] < 0.f) {
      return fail(DORT_ERR_INVALID, "tri_albedo must be finite and non-negative");
    }
  }
  for(size_t i = 0; emission && i < n; ++i) {
    if(!std::isfinite(emission[i]) || emission[i] < 0.f) {
      return fail(DORT_ERR_INVALID, "tri_emission must be finite and non-negative");
    }
  }
  auto put = [&](const float* src, float** buf, const float** view) -> int {
    if(!src) { *view = nullptr; return DORT_OK; }
    if(!*buf) {
      void* d = nullptr;
      if(dev_alloc(&d, bytes ? bytes : 4) != cudaSuccess) {
        cudaGetLastError();
        return fail(DORT_ERR_OOM, "cudaMalloc of triangle parameters failed");
      }
      s->allocations.push_back(d);
      s->device_bytes += bytes;
      *buf = static_cast<float*>(d);
    }
    DG_CUDA(cudaMemcpy(*buf, src, bytes, cudaMemcpyHostToDevice));
    *view = *buf;
    return DORT_OK;
  };
  int rc = put(albedo, &s->d_tri_albedo, &s->pt.tri_albedo);
  if(rc != DORT_OK) { return rc; }
  return put(emission, &s->d_tri_emission, &s->pt.tri_emission);
}

}  // namespace dort_gpu

using namespace dort_gpu;

extern "C" int dort_gpu_adjoint_forward(dort_scene* scene, const dort_render_params* params,
                                        const float* tri_albedo, const float* tri_emission,
                                        float* out_image) try {
  clear_error();
  if(!scene || !params || !out_image) { return fail(DORT_ERR_INVALID, "null argument"); }
  int rc = require_scene_device(scene);
  if(rc != DORT_OK) { return rc; }
  rc = set_tri_params(scene, tri_albedo, tri_emission);
  if(rc != DORT_OK) { return rc; }
  // the path tracer renders as a wavefront whose sums are added in a fixed
  // order, so that the same parameters give the same image (finite
  // differences of the loss rely on it); DORT_ADJOINT_MEGAKERNEL keeps the
  // megakernel, the other renderers render as dort_gpu_render does
  if(params->renderer == DORT_RENDERER_PT && params->struct_size == sizeof(dort_render_params) &&
     !(params->renderer_flags & DORT_ADJOINT_MEGAKERNEL)) {
    dort_wavefront_tuning t{};
    t.struct_size = sizeof(t);
    t.deterministic = 1;
    return dort_gpu_render_wavefront(scene, params, &t, out_image, nullptr);
  }
  return dort_gpu_render(scene, params, out_image, nullptr);
} DORT_ABI_CATCH

extern "C" int dort_gpu_adjoint_backward(dort_scene* scene, const dort_render_params* params,
                                         const float* tri_albedo, const float* tri_emission,
                                         const float* dl_dimage, float* d_albedo,
                                         float* d_emission) try {
  clear_error();
  if(!scene || !params || !dl_dimage || (!d_albedo && !d_emission)) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  PtParams pp;
  std::string err;
  if(!make_params(params, pp, err)) { return fail(DORT_ERR_INVALID, err); }
  if(pp.renderer != RENDERER_PT) {
    return fail(DORT_ERR_UNSUPPORTED, "the adjoint renders only the pt renderer");
  }
  int rc = require_scene_device(scene);
  if(rc != DORT_OK) { return rc; }
  rc = set_tri_params(scene, tri_albedo, tri_emission);
  if(rc != DORT_OK) { return rc; }
  if(d_emission && !scene->pt.tri_emission) {
    return fail(DORT_ERR_INVALID, "emission gradients need tri_emission");
  }
  size_t npix = size_t(pp.width) * pp.height;
  size_t tbytes = size_t(scene->tri_count) * 3 * sizeof(float);
  const bool megakernel = (params->renderer_flags & DORT_ADJOINT_MEGAKERNEL) != 0;
  // the wavefront's path slots: one per 4-sample work unit, at most 2^22
  const uint64_t units = uint64_t((pp.width + 7) / 8) * ((pp.height + 3) / 4) * 32 *
                         ((uint64_t(pp.spp) + 3) / 4);
  const uint32_t capacity = uint32_t((std::min<uint64_t>(units, kAdjSlots) + 31) & ~uint64_t(31));
  // samples whose terms overflow the wavefront's log, traced again: a list
  // of up to every sample of the frame, at most 2^24
  uint32_t overflow_cap = uint32_t(std::min<uint64_t>(uint64_t(npix) * pp.spp, kAdjListMax));
  const long long cap_override = g_adj_list_cap.load();
  if(cap_override >= 0) { overflow_cap = uint32_t(std::min<long long>(cap_override, overflow_cap)); }
  // dLoss/dimage, the albedo and emission gradients, the overflow list and
  // its count, in one grow-only buffer held by the scene (256-byte aligned)
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t img_bytes = align(npix * 3 * sizeof(float)), tri_bytes = align(tbytes);
  const size_t list_bytes = align(size_t(overflow_cap) * sizeof(uint2));
  const size_t need = img_bytes + 2 * tri_bytes + list_bytes + 256;
  if(scene->adjoint_bytes < need) {
    if(scene->d_adjoint) { cudaFree(scene->d_adjoint); }
    scene->d_adjoint = nullptr;
    scene->adjoint_bytes = 0;
    if(dev_alloc(&scene->d_adjoint, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(DORT_ERR_OOM, "cudaMalloc for the adjoint failed");
    }
    scene->adjoint_bytes = need;
  }
  char* base = static_cast<char*>(scene->d_adjoint);
  float* d_img = reinterpret_cast<float*>(base);
  float* d_ga = d_albedo ? reinterpret_cast<float*>(base + img_bytes) : nullptr;
  float* d_ge = d_emission ? reinterpret_cast<float*>(base + img_bytes + tri_bytes) : nullptr;
  uint2* d_list = reinterpret_cast<uint2*>(base + img_bytes + 2 * tri_bytes);
  uint32_t* d_list_n = reinterpret_cast<uint32_t*>(base + img_bytes + 2 * tri_bytes + list_bytes);
  cudaStream_t st = 0;
  auto zero_gradients = [&]() {
    bool z = true;
    if(d_ga) { z = z && cudaMemsetAsync(d_ga, 0, tbytes, st) == cudaSuccess; }
    if(d_ge) { z = z && cudaMemsetAsync(d_ge, 0, tbytes, st) == cudaSuccess; }
    return z;
  };
  bool ok = cudaMemcpyAsync(d_img, dl_dimage, npix * 3 * sizeof(float),
                            cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && zero_gradients();
  const bool general = scene_needs_general(scene->pt, pp);
  // the megakernel form: one thread per (pixel, slice of samples)
  auto run_megakernel = [&]() -> int {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    MegaPlan plan;
    if(megakernel_plan(scene->device, dev, sms, pp.width, pp.height, pp.spp, 0, &plan) != 0) {
      return fail(DORT_ERR_INVALID, plan.why);
    }
    const uint64_t threads = uint64_t(plan.slices) * plan.per_slice;
    const uint32_t grid = uint32_t((threads + kAdjBlock - 1) / kAdjBlock);
    if(general) {
      adjoint_replay<true><<<grid, kAdjBlock, 0, st>>>(scene->pt, pp, plan.slices, plan.per,
                                                         plan.per_slice, d_img, d_ga, d_ge);
    } else {
      adjoint_replay<false><<<grid, kAdjBlock, 0, st>>>(scene->pt, pp, plan.slices, plan.per,
                                                          plan.per_slice, d_img, d_ga, d_ge);
    }
    return cudaGetLastError() == cudaSuccess ? DORT_OK
                                             : fail(DORT_ERR_CUDA, "adjoint launch failed");
  };
  for(double& v : scene->adjoint_stats) { v = 0.0; }
  if(ok && megakernel) {
    scene->adjoint_stats[0] = 1.0;
    rc = run_megakernel();
    if(rc != DORT_OK) { return rc; }
  } else if(ok) {
    ok = cudaMemsetAsync(d_list_n, 0, sizeof(uint32_t), st) == cudaSuccess;
    WfTuning tn{};
    tn.capacity = capacity;
    tn.trace_block = 128;
    tn.shade_block = 128;
    if(ok) {
      rc = wavefront_adjoint(scene, pp, tn, d_img, d_ga, d_ge, d_list, overflow_cap, d_list_n,
                             st);
      if(rc != DORT_OK) { return rc; }
    }
    uint32_t listed = 0;
    ok = ok && cudaMemcpyAsync(&listed, d_list_n, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if(ok) {
      uint64_t rays = 0;
      uint32_t waves = 0, error = 0;
      rc = wavefront_adjoint_counters(scene, &rays, &waves, &error, st);
      if(rc != DORT_OK) { return rc; }
      if(error) {
        return fail(DORT_ERR_TIMEOUT, "the adjoint's wavefront reached its wave bound");
      }
      scene->adjoint_stats[1] = double(listed);
      scene->adjoint_stats[2] = double(rays);
      scene->adjoint_stats[3] = double(waves);
    }
    if(ok && listed > overflow_cap) {
      // more overflowing samples than the list holds: the megakernel form
      // for every sample instead
      scene->adjoint_stats[0] = 2.0;
      ok = zero_gradients();
      if(ok) {
        rc = run_megakernel();
        if(rc != DORT_OK) { return rc; }
      }
    } else if(ok && listed > 0) {
      const uint32_t grid = (listed + kAdjBlock - 1) / kAdjBlock;
      if(general) {
        adjoint_replay_list<true><<<grid, kAdjBlock, 0, st>>>(scene->pt, pp, d_list, listed,
                                                                d_img, d_ga, d_ge);
      } else {
        adjoint_replay_list<false><<<grid, kAdjBlock, 0, st>>>(scene->pt, pp, d_list, listed,
                                                                 d_img, d_ga, d_ge);
      }
      ok = cudaGetLastError() == cudaSuccess;
    }
  }
  if(ok && d_albedo) {
    ok = cudaMemcpyAsync(d_albedo, d_ga, tbytes, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  }
  if(ok && d_emission) {
    ok = cudaMemcpyAsync(d_emission, d_ge, tbytes, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  }
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  if(!ok) {
    return fail(DORT_ERR_CUDA, std::string("adjoint failed: ") +
                               cudaGetErrorString(cudaGetLastError()));
  }
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_debug_adjoint_list(long long entries) try {
  clear_error();
  g_adj_list_cap.store(entries < 0 ? -1 : entries);
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_adjoint_stats(dort_scene* scene, double* out_stats) try {
  clear_error();
  if(!scene || !out_stats) { return fail(DORT_ERR_INVALID, "null argument"); }
  for(int k = 0; k < 4; ++k) { out_stats[k] = scene->adjoint_stats[k]; }
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_loss_l2(const float* image, const float* target, size_t count,
                                double* out_loss, float* out_grad) try {
  clear_error();
  if(!image || !target || !out_loss || !out_grad) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  if(count > 0xffffffffull) { return fail(DORT_ERR_INVALID, "count exceeds 2^32 - 1"); }
  // image, target and gradient (256-byte aligned) and the loss, in a
  // grow-only buffer per device kept for the process; one call at a time
  static std::mutex mu;
  static std::vector<std::pair<void*, size_t>> scratch;
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  if(scratch.size() <= size_t(dev)) { scratch.resize(size_t(dev) + 1, {nullptr, 0}); }
  size_t bytes = count * sizeof(float);
  const size_t part = (bytes + 255) & ~size_t(255);
  const size_t need = 3 * part + sizeof(double);
  auto& buf = scratch[size_t(dev)];
  if(buf.second < need) {
    if(buf.first) { cudaFree(buf.first); }
    buf = {nullptr, 0};
    if(dev_alloc(&buf.first, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(DORT_ERR_OOM, "cudaMalloc for the loss failed");
    }
    buf.second = need;
  }
  char* base = static_cast<char*>(buf.first);
  float* d_a = reinterpret_cast<float*>(base);
  float* d_b = reinterpret_cast<float*>(base + part);
  float* d_g = reinterpret_cast<float*>(base + 2 * part);
  double* d_l = reinterpret_cast<double*>(base + 3 * part);
  bool ok = true;
  cudaStream_t st = 0;
  ok = ok && cudaMemcpyAsync(d_a, image, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(d_b, target, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemsetAsync(d_l, 0, sizeof(double), st) == cudaSuccess;
  if(ok && count) {
    l2_loss_grad<<<uint32_t((count + 255) / 256), 256, 0, st>>>(d_a, d_b, uint32_t(count), d_g,
                                                                  d_l);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && cudaMemcpyAsync(out_grad, d_g, bytes, cudaMemcpyDeviceToHost, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(out_loss, d_l, sizeof(double), cudaMemcpyDeviceToHost, st) ==
                 cudaSuccess;
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  if(!ok) {
    cudaGetLastError();
    return fail(DORT_ERR_CUDA, "l2 loss failed");
  }
  return DORT_OK;
} DORT_ABI_CATCH
