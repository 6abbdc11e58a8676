// Wavefront path tracer: the paths of PathRenderer::sample
// (path_renderer.cpp:23-111) split into stages that run over device-resident
// queues, one wave (one bounce of every live path) at a time:
//
//   regen   finished paths -> film; free slots take the next sample (path
//           regeneration); live slots are compacted into the active queue
//   extend  closest hit of every active path's ray
//   shade   emission, direct-lighting setup (one shadow ray and one
//           BSDF-strategy ray per path into two queues), continuation
//           sample, Russian roulette
//   shadow  any hit of the shadow queue; unoccluded contributions added
//   neeb    closest hit of the BSDF-strategy queue; light hits added with
//           their MIS weight
//   control resets the queue counters and sets the loop condition
//
// The waves run inside one CUDA graph per frame: a conditional while node
// whose body holds the six kernels, so the host launches a frame once.
// Queues are compacted with warp ballots (one atomic per warp).  Every kernel
// is a grid-stride loop over a count it reads from device memory, so the
// graph's launch shapes are fixed.
//
// Random numbers are the megakernel's (philox.cuh, keyed by pixel, sample and
// bounce), so both renderers trace the same paths; only the order of film
// additions (float atomics here) differs.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <string>

#include "adjoint.cuh"
#include "autotune_plan.h"
#include "common.h"
#include "pt.cuh"
#include "scene_build.h"
#include "wavefront.h"

namespace dort_gpu {

enum : uint32_t { SLOT_FREE = 0, SLOT_ACTIVE = 1, SLOT_FINISHED = 2 };

// Device counters.  Queues that are produced in one wave and consumed in the
// next are double-buffered; buffer b of wave w is (w + b) & 1.
enum : uint32_t {
  C_ACT0 = 0, C_ACT1 = 1,      // active queue lengths (per buffer)
  C_FIN0 = 2, C_FIN1 = 3,      // finished queue lengths (per buffer)
  C_SHADOW = 4, C_NEEB = 5,    // this wave's shadow / BSDF-strategy queues
  C_LIVE = 6, C_WAVES = 7, C_ERROR = 8,
  C_F_EXT = 9, C_F_SHADE = 10, C_F_SH = 11, C_F_NB = 12,   // work-fetch cursors
  C_KQ0 = 20,       // [20..25]: lengths of the shade queues by material kind
  C_NEXT_LO = 16,   // 64-bit next-sample counter at [16..17]
  C_RAYS_LO = 18,   // 64-bit ray counter at [18..19]
  C_COUNT = 32
};

// Each counter sits alone at the start of a 128-byte line (a 64-bit counter
// takes the line's first two words): the stages' warp-aggregated atomics on
// different counters then go to different L2 lines instead of queueing on
// one.
constexpr uint32_t kCtrStride = 32;

DG_HD uint32_t* ctr_at(uint32_t* ctr, uint32_t i) { return ctr + i * kCtrStride; }

// Shade queues: paths are sorted by what they hit (material kind 0..4, or a
// miss) so that the warps of the shade stage run one BSDF's code.
constexpr uint32_t kShadeQueues = 6;
constexpr uint32_t kMissQueue = 5;

DG_HD uint32_t f2u(float f) { return DG_AS_UINT(f); }
DG_HD float u2f(uint32_t u) { return DG_AS_FLOAT(u); }

// Warp-aggregated append: returns this lane's index in the queue.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  uint32_t mask = __ballot_sync(0xffffffffu, want);
  if(!want) { return 0; }
  uint32_t lane = threadIdx.x & 31u;
  uint32_t leader = __ffs(mask) - 1u;
  uint32_t base = 0;
  if(lane == leader) { base = atomicAdd(counter, __popc(mask)); }
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

// Next 32 work items for this warp from a fetch cursor (lane 0 advances it).
__device__ __forceinline__ uint32_t warp_fetch(uint32_t* cursor) {
  uint32_t base = 0;
  if((threadIdx.x & 31u) == 0) { base = atomicAdd(cursor, 32u); }
  return __shfl_sync(0xffffffffu, base, 0);
}

// Work is handed out in units of kChunk consecutive samples of one pixel:
// the path slot that takes a unit traces its samples one after the other and
// adds their sum to the film once.  Unit ids run chunk-major over 8x4 pixel
// tiles, so consecutive units are neighbouring pixels (coherent primary rays).
// One sample per unit measured fastest once the frame holds enough path
// slots (2^27: a quarter of the 1080p frame's samples in flight): every
// finished sample's slot takes the next sample in tile order, so the waves
// stay full and their primary rays coherent.  1080p frame 725.8 / 698.2 /
// 670.3 / 626.9 M samples/s with 1 / 2 / 4 / 8 samples per unit; Cornell
// workload 1,097 / 973 / 869 M; adjoint 132 / 142 / 157 ms.
constexpr uint32_t kChunk = kWfUnitSamples;

__device__ __forceinline__ void unit_to_pixel(const PtParams& pp, uint64_t uid, uint32_t& pixel,
                                              uint32_t& x, uint32_t& y, uint32_t& s0) {
  uint32_t tiles_x = (pp.width + 7) / 8;
  uint32_t tiles = tiles_x * ((pp.height + 3) / 4);
  uint64_t per_chunk = uint64_t(tiles) * 32;
  uint32_t c = uint32_t(uid / per_chunk);
  uint32_t local = uint32_t(uid % per_chunk);
  uint32_t tile = local / 32, lane = local % 32;
  x = (tile % tiles_x) * 8 + lane % 8;
  y = (tile / tiles_x) * 4 + lane / 8;
  pixel = y * pp.width + x;
  s0 = c * kChunk;
}

struct WfDev {
  float4* ray_o;   // o.xyz, t_min
  float4* ray_d;   // d.xyz, -
  float4* thr;     // throughput
  float4* sum;     // radiance sum of the current path
  float4* acc;     // kept samples of the slot's unit: sum rgb, count
  uint4* meta;     // pixel, sample, bounces | last_delta << 31, state | job << 8
  float4* hit;     // t, b1, b2, prim
  uint32_t* active[2];
  uint32_t* finished[2];
  uint32_t* kq[kShadeQueues];   // shade queues by hit kind
  uint32_t* sh_slot;
  float4* sh_o;    // o.xyz, t_min
  float4* sh_d;    // d.xyz, t_max
  float4* sh_c;    // contribution
  uint32_t* nb_slot;
  float4* nb_o;    // o.xyz, t_min
  float4* nb_d;    // d.xyz, pdf
  float4* nb_f;    // factor.xyz, light index (bits) | use_mis << 31
  float4* film;    // sum rgb, kept count
  uint32_t* sort_key[2];   // ray sort: keys in / out (capacity each)
  uint32_t* sort_val[2];   // slots in (the active queue's order) / out (sorted)
  uint32_t* hit_kind;      // per slot: shade queue of the hit (sorted extension)
  void* sort_temp;         // CUB temporary storage
  size_t sort_temp_bytes;
  uint32_t sorted;         // 1: the extension stage traces in sorted order
  uint32_t* ctr;
  uint32_t capacity;
  uint64_t total_samples;   // work units (see kChunk) of all jobs
  uint32_t max_waves;
  // the adjoint's term log (adjoint.cuh): entry k of slot s at
  // adj_log[k * capacity + s], adj_n[s] entries so far (above kAdjLog: the
  // sample overflowed); null outside the adjoint
  float4* adj_log;
  uint32_t* adj_n;
  // deterministic sums (single frames): the sum of work unit u of pixel p at
  // unit_film[u * npix + p], added in unit order by the resolve; null: the
  // units are added to film by atomics
  float4* unit_film;
  uint32_t npix;
};

// Where a path's scene and render parameters come from.  A single frame
// passes them as kernel arguments; a batch of frames (many scenes, each with
// its own resolution, spp and depth) reads a device table of jobs, and every
// path carries its job index in the high bits of meta.w.
// G selects the instantiation of the path code (pt.cuh).
template<bool G>
struct SingleJob {
  static constexpr bool kBatched = false;
  static constexpr bool kGeneral = G;
  static constexpr bool kAdjoint = false;
  PtScene sc;
  PtParams pp;
  __device__ __forceinline__ uint32_t job_of_sample(uint64_t) const { return 0; }
  __device__ __forceinline__ uint64_t sample_begin(uint32_t) const { return 0; }
  __device__ __forceinline__ const PtScene& scene(uint32_t) const { return sc; }
  __device__ __forceinline__ const PtParams& params(uint32_t) const { return pp; }
  __device__ __forceinline__ uint32_t film_offset(uint32_t) const { return 0; }
};

struct WfJob {
  PtScene sc;
  PtParams pp;
  uint64_t sample_begin;   // first global work-unit id of the job
  uint32_t film_offset;    // first pixel of the job in the batch film
  uint32_t pad;
};

template<bool G>
struct JobTable {
  static constexpr bool kBatched = true;
  static constexpr bool kGeneral = G;
  static constexpr bool kAdjoint = false;
  const WfJob* jobs;
  uint32_t count;
  __device__ __forceinline__ uint32_t job_of_sample(uint64_t sid) const {
    uint32_t lo = 0, hi = count;         // last job with sample_begin <= sid
    while(lo + 1 < hi) {
      uint32_t mid = (lo + hi) / 2;
      if(jobs[mid].sample_begin <= sid) { lo = mid; } else { hi = mid; }
    }
    return lo;
  }
  __device__ __forceinline__ uint64_t sample_begin(uint32_t j) const { return jobs[j].sample_begin; }
  __device__ __forceinline__ const PtScene& scene(uint32_t j) const { return jobs[j].sc; }
  __device__ __forceinline__ const PtParams& params(uint32_t j) const { return jobs[j].pp; }
  __device__ __forceinline__ uint32_t film_offset(uint32_t j) const { return jobs[j].film_offset; }
};

// The backward pass of the adjoint as a wavefront: a single frame whose
// paths record their terms in the slot's log (shade: emission and Lambert
// vertices; shadow and BSDF-strategy stages: direct-lighting terms from
// light triangles) and whose regeneration stage turns a finished sample's
// log into gradients.  Samples whose terms overflow the log are listed as
// (pixel, sample) for a second trace (adjoint.cu).
template<bool G>
struct AdjointJob : SingleJob<G> {
  static constexpr bool kAdjoint = true;
  const float* dl_dimage;   // dLoss/dI (width * height * 3)
  float* d_albedo;          // gradients (tri_count * 3 each), either may be null
  float* d_emission;
  uint2* overflow;          // (pixel, sample) of the samples that overflowed
  uint32_t* overflow_n;     // their count (may exceed overflow_cap: then all are lost)
  uint32_t overflow_cap;
};

// One log entry of `slot` (entries = 1, or 2 for a vertex); the stages that
// may append to a slot concurrently (several shadow entries per path) pass
// atomic.
template<bool ATOMIC>
__device__ __forceinline__ uint32_t adj_reserve(WfDev& w, uint32_t slot, uint32_t entries) {
  if(ATOMIC) { return atomicAdd(&w.adj_n[slot], entries); }
  const uint32_t k = w.adj_n[slot];
  w.adj_n[slot] = k + entries;
  return k;
}

template<bool ATOMIC>
__device__ __forceinline__ void adj_record(WfDev& w, uint32_t slot, uint32_t kind,
                                           uint32_t prim, V3 v) {
  // a primitive index that does not fit the tag overflows the sample
  const uint32_t k = adj_reserve<ATOMIC>(w, slot, prim > kEvPrimMask ? kAdjLog + 1 : 1u);
  if(prim <= kEvPrimMask && k < kAdjLog) {
    w.adj_log[size_t(k) * w.capacity + slot] = adj_entry(kind, prim, v);
  }
}

__device__ __forceinline__ uint32_t wave_of(const WfDev& w) {
  return *(volatile uint32_t*)ctr_at(w.ctr, C_WAVES);
}

__global__ void wf_init(WfDev w, uint32_t npix) {
  uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < w.capacity; i += stride) {
    w.meta[i] = make_uint4(0u, 0u, 0u, SLOT_FREE);
    w.finished[0][i] = uint32_t(i);    // every slot starts on the free list
    if(w.adj_n) { w.adj_n[i] = 0u; }
  }
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < npix; i += stride) {
    w.film[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if(blockIdx.x == 0) {
    for(uint32_t i = threadIdx.x; i < C_COUNT * kCtrStride; i += blockDim.x) {
      w.ctr[i] = i == C_FIN0 * kCtrStride ? w.capacity : 0u;
    }
  }
}

// Direction octant of a ray (sign bits of x, y, z).  The path state keeps
// the octant of its next extension ray in bits 28..30 of meta.z (bounces
// take the bits below: max_depth <= 1000), so that regen can group the
// active queue by octant without reading the rays.
constexpr uint32_t kOctShift = 28;
constexpr uint32_t kBounceMask = (1u << kOctShift) - 1u;

DG_HD uint32_t dir_octant(V3 d) {
  return (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
}

// Starts sample s of `pixel` in `slot`: camera ray, unit throughput.
// Returns the camera ray's direction octant.
template<bool G>
__device__ __forceinline__ uint32_t start_path(WfDev& w, const PtParams& pp, uint32_t slot,
                                               uint32_t pixel, uint32_t s) {
  uint32_t x = pixel % pp.width, y = pixel / pp.width;
  float fx, fy;
  if(s == 0) {
    fx = float(x) + 0.5f;
    fy = float(y) + 0.5f;
  } else {
    Rand4 j = rand4(pp.seed, pixel, s, kBlockCamera);
    fx = float(x) + j.a;
    fy = float(y) + j.b;
  }
  V3 o, d;
  camera_ray<G>(pp, pixel, s, fx, fy, o, d);
  w.ray_o[slot] = make_float4(o.x, o.y, o.z, 0.f);
  w.ray_d[slot] = make_float4(d.x, d.y, d.z, 0.f);
  w.thr[slot] = make_float4(1.f, 1.f, 1.f, 0.f);
  w.sum[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
  return dir_octant(d);
}

// Builds this wave's active queue.  It walks the previous wave's active queue
// in order: continuing paths stay; a finished path's sample joins its slot's
// unit sum and the slot starts the unit's next sample in the same place, or,
// when the unit is done, adds the unit to the film and takes a new unit.  Then
// it walks the free list (every slot in the first wave; slots whose unit fell
// outside the image later).  Keeping the queue order keeps neighbouring
// pixels' primary rays next to each other whatever order the shade stage ran
// the paths in.
// Block-wide counts of the regen stage: per warp, then one atomic per block
// and counter (the stage's appends would otherwise queue one atomic per warp
// on the same counters).  kRegenBlock threads, every thread of a block takes
// part in every round.
constexpr uint32_t kRegenBlock = 256;
constexpr uint32_t kRegenWarps = kRegenBlock / 32;

struct RegenShared {
  uint32_t cnt[3][kRegenWarps];   // per warp: new units, (unused), free appends
  int live[kRegenWarps];          // per warp: change of the live-unit count
  unsigned long long next_base;
  uint32_t base[2];
  uint32_t oc[8][kRegenWarps];    // per direction octant and warp: active appends
};

// Exclusive scan of cnt[k] over the warps (thread 0); returns the total.
__device__ __forceinline__ uint32_t regen_scan(uint32_t* cnt) {
  uint32_t t = 0;
  for(uint32_t w = 0; w < kRegenWarps; ++w) {
    uint32_t c = cnt[w];
    cnt[w] = t;
    t += c;
  }
  return t;
}

// The end of a sample in the adjoint's backward pass: its log becomes
// gradients (samples the film drops have none), or the sample is listed for
// a second trace when its terms overflowed the log; the log is emptied for
// the slot's next sample.
template<class J>
__device__ __forceinline__ void adj_finish(const J& jobs, WfDev& w, uint32_t slot,
                                           uint32_t pixel, uint32_t sample, V3 L) {
  const uint32_t n = w.adj_n[slot];
  w.adj_n[slot] = 0u;
  if(n == 0u || !adj_kept(L)) { return; }
  const float inv_spp = 1.f / float(jobs.pp.spp);
  const V3 adj = v3(jobs.dl_dimage[3 * size_t(pixel)], jobs.dl_dimage[3 * size_t(pixel) + 1],
                    jobs.dl_dimage[3 * size_t(pixel) + 2]) * inv_spp;
  if(is_black(adj)) { return; }
  if(n > kAdjLog) {
    const uint32_t k = atomicAdd(jobs.overflow_n, 1u);
    if(k < jobs.overflow_cap) { jobs.overflow[k] = make_uint2(pixel, sample); }
    return;
  }
  adj_apply(w.adj_log + slot, w.capacity, n, L, adj, jobs.sc.tri_emission, jobs.d_albedo,
            jobs.d_emission);
}

template<class J>
__device__ __forceinline__ void regen_slot(J& jobs, WfDev& w, bool valid, uint32_t slot,
                                           uint32_t cur, bool from_free, RegenShared& sh) {
  uint64_t* next = reinterpret_cast<uint64_t*>(ctr_at(w.ctr, C_NEXT_LO));
  uint32_t* act = w.active[cur];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  uint4 m = valid ? w.meta[slot] : make_uint4(0u, 0u, 0u, SLOT_FREE + 7u);
  bool keep = valid && (m.w & 0xffu) == SLOT_ACTIVE && !from_free;
  bool started = false;
  int live = 0;
  uint32_t oct = (m.z >> kOctShift) & 7u;
  if(valid && (m.w & 0xffu) == SLOT_FINISHED) {
    const uint32_t job = m.w >> 8;
    const PtParams& pp = jobs.params(job);
    float4 s = w.sum[slot];
    float4 a = w.acc[slot];
    // renderer.cpp:36-41: only finite, non-negative samples reach the film
    if(isfinite(s.x) && isfinite(s.y) && isfinite(s.z) && s.x >= 0.f && s.y >= 0.f &&
       s.z >= 0.f) {
      a = make_float4(a.x + s.x, a.y + s.y, a.z + s.z, a.w + 1.f);
    }
    if constexpr(J::kAdjoint) { adj_finish(jobs, w, slot, m.x, m.y, v3(s.x, s.y, s.z)); }
    uint32_t next_s = m.y + 1u;
    uint32_t unit_end = min(pp.spp, (m.y / kChunk + 1u) * kChunk);
    if(next_s < unit_end) {
      w.acc[slot] = a;
      oct = start_path<J::kGeneral>(w, pp, slot, m.x, next_s);
      m = make_uint4(m.x, next_s, oct << kOctShift, SLOT_ACTIVE | (job << 8));
      started = true;
    } else {
      if(!J::kBatched && w.unit_film) {
        w.unit_film[size_t(m.y / kChunk) * w.npix + m.x] = a;
      } else if(a.w > 0.f || a.x != 0.f || a.y != 0.f || a.z != 0.f) {
        atomicAdd(w.film + jobs.film_offset(job) + m.x, a);
      }
      live -= 1;
      m.w = SLOT_FREE;
    }
  }
  // new units: one 64-bit atomic per block on the next-unit counter
  bool want_new = valid && (m.w & 0xffu) == SLOT_FREE;
  uint32_t nmask = __ballot_sync(0xffffffffu, want_new);
  if(lane == 0) { sh.cnt[0][warp] = __popc(nmask); }
  __syncthreads();
  if(threadIdx.x == 0) {
    uint32_t t = regen_scan(sh.cnt[0]);
    sh.next_base = t ? atomicAdd(reinterpret_cast<unsigned long long*>(next),
                                 (unsigned long long)t) : 0ull;
  }
  __syncthreads();
  uint64_t uid = want_new ? sh.next_base + sh.cnt[0][warp] + __popc(nmask & lt) : ~0ull;
  if(want_new && uid < w.total_samples) {
    uint32_t job = jobs.job_of_sample(uid);
    const PtParams& pp = jobs.params(job);
    uint32_t pixel, x, y, s0;
    unit_to_pixel(pp, uid - jobs.sample_begin(job), pixel, x, y, s0);
    if(x < pp.width && y < pp.height) {
      w.acc[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
      oct = start_path<J::kGeneral>(w, pp, slot, pixel, s0);
      m = make_uint4(pixel, s0, oct << kOctShift, SLOT_ACTIVE | (job << 8));
      started = true;
      live += 1;
    }
  }
  if(valid && (started || want_new)) { w.meta[slot] = m; }
  // a slot whose unit fell outside the image goes on the next free list so
  // that it keeps taking units
  bool retry = want_new && !started && uid < w.total_samples;
  bool put = keep || started;
  // the active queue is grouped by direction octant within each block's
  // share (slot order kept within an octant): the extension stage's warps
  // then take rays that visit a node's children in the same order
  uint32_t omask = 0u;
#pragma unroll
  for(uint32_t k = 0; k < 8u; ++k) {
    uint32_t mk = __ballot_sync(0xffffffffu, put && oct == k);
    if(lane == 0) { sh.oc[k][warp] = __popc(mk); }
    if(oct == k) { omask = mk; }
  }
  uint32_t rmask = __ballot_sync(0xffffffffu, retry);
  int wlive = __reduce_add_sync(0xffffffffu, live);
  if(lane == 0) {
    sh.cnt[2][warp] = __popc(rmask);
    sh.live[warp] = wlive;
  }
  __syncthreads();
  if(threadIdx.x == 0) {
    // exclusive scan in (octant, warp) order
    uint32_t ta = 0;
    for(uint32_t k = 0; k < 8u; ++k) {
      for(uint32_t q = 0; q < kRegenWarps; ++q) {
        uint32_t c = sh.oc[k][q];
        sh.oc[k][q] = ta;
        ta += c;
      }
    }
    uint32_t tr = regen_scan(sh.cnt[2]);
    int tl = 0;
    for(uint32_t k = 0; k < kRegenWarps; ++k) { tl += sh.live[k]; }
    sh.base[0] = ta ? atomicAdd(ctr_at(w.ctr, C_ACT0 + cur), ta) : 0u;
    sh.base[1] = tr ? atomicAdd(ctr_at(w.ctr, C_FIN0 + (cur ^ 1u)), tr) : 0u;
    if(tl != 0) { atomicAdd(ctr_at(w.ctr, C_LIVE), uint32_t(tl)); }
  }
  __syncthreads();
  if(put) { act[sh.base[0] + sh.oc[oct][warp] + __popc(omask & lt)] = slot; }
  if(retry) { w.finished[cur ^ 1u][sh.base[1] + sh.cnt[2][warp] + __popc(rmask & lt)] = slot; }
}

template<class J>
__global__ void __launch_bounds__(kRegenBlock) wf_regen(J jobs, WfDev w) {
  __shared__ RegenShared sh;
  const uint32_t wave = wave_of(w);
  const uint32_t cur = wave & 1u, prev = cur ^ 1u;
  const uint32_t n_prev = *(volatile uint32_t*)ctr_at(w.ctr, C_ACT0 + prev);
  const uint32_t n_free = *(volatile uint32_t*)ctr_at(w.ctr, C_FIN0 + cur);
  const uint32_t* old = w.active[prev];
  const uint32_t* fre = w.finished[cur];
  // every thread of a block runs the same number of iterations (the rounds
  // of regen_slot synchronise the block)
  const uint32_t stride = gridDim.x * kRegenBlock;
  const uint32_t np = (n_prev + kRegenBlock - 1u) / kRegenBlock * kRegenBlock;
  for(uint32_t i = blockIdx.x * kRegenBlock + threadIdx.x; i < np; i += stride) {
    bool valid = i < n_prev;
    regen_slot(jobs, w, valid, valid ? old[i] : 0u, cur, false, sh);
  }
  const uint32_t nf = (n_free + kRegenBlock - 1u) / kRegenBlock * kRegenBlock;
  for(uint32_t i = blockIdx.x * kRegenBlock + threadIdx.x; i < nf; i += stride) {
    bool valid = i < n_free;
    regen_slot(jobs, w, valid, valid ? fre[i] : 0u, cur, true, sh);
  }
}

// Ray sort before the extension stage: key = direction octant (3 bits) and
// the Morton code of the origin's cell on a 32^3 grid over the scene's
// bounding cube (15 bits).  The sort is stable, so primary rays (one origin
// for a pinhole) keep their pixel order within an octant.  Every wave sorts
// the whole queue capacity (the graph is built once; the length lives on the
// device): positions past the active length get the largest key and stay
// behind the rays.
constexpr int kSortBits = 18;

__device__ __forceinline__ uint32_t spread5(uint32_t v) {
  uint32_t r = 0;
#pragma unroll
  for(int b = 0; b < 5; ++b) { r |= ((v >> b) & 1u) << (3 * b); }
  return r;
}

__device__ __forceinline__ uint32_t cell_of(float x, float lo, float inv) {
  float f = (x - lo) * inv;
  return f <= 0.f ? 0u : (f >= 31.f ? 31u : uint32_t(f));
}

template<class J>
__global__ void wf_sort_keys(J jobs, WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  const uint32_t n = *(volatile uint32_t*)ctr_at(w.ctr, C_ACT0 + cur);
  const uint32_t* act = w.active[cur];
  for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.capacity;
      i += gridDim.x * blockDim.x) {
    uint32_t key = (1u << kSortBits) - 1u, val = 0u;
    if(i < n) {
      val = act[i];
      uint32_t job = J::kBatched ? (w.meta[val].w >> 8) : 0u;
      const PtScene& sc = jobs.scene(job);
      float4 o = w.ray_o[val], d = w.ray_d[val];
      float r = sc.radius;
      float inv = r > 0.f ? 16.f / r : 0.f;   // 32 cells over 2r
      uint32_t m = spread5(cell_of(o.x, sc.centroid[0] - r, inv)) |
                   (spread5(cell_of(o.y, sc.centroid[1] - r, inv)) << 1) |
                   (spread5(cell_of(o.z, sc.centroid[2] - r, inv)) << 2);
      uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
      key = (oct << 15) | m;
    }
    w.sort_key[0][i] = key;
    w.sort_val[0][i] = val;
  }
}

// After a sorted extension: the shade queues in the active queue's own order,
// so that the shade stage and the next regeneration walk the path slots as
// they did unsorted (mostly ascending, coalesced) rather than in ray order.
__global__ void wf_classify(WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  const uint32_t n = *(volatile uint32_t*)ctr_at(w.ctr, C_ACT0 + cur);
  const uint32_t* act = w.active[cur];
  uint32_t np = (n + 31u) & ~31u;
  for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    uint32_t slot = 0, kind = kShadeQueues;
    if(i < n) {
      slot = act[i];
      kind = w.hit_kind[slot];
    }
#pragma unroll
    for(uint32_t k = 0; k < kShadeQueues; ++k) {
      bool mine = kind == k;
      uint32_t at = warp_append(ctr_at(w.ctr, C_KQ0 + k), mine);
      if(mine) { w.kq[k][at] = slot; }
    }
  }
}

// Register cap of the trace stages (extend, shadow): 56 instead of the 64
// the compiler picks (a few bytes of spill) lets 9 instead of 8 blocks of 128
// threads share an SM; the 1080p frame measured 659.7 against 652.2 M
// samples/s (extend 338.9 against 345.4 ms).
#ifndef DORT_TRACE_MAXNREG
#define DORT_TRACE_MAXNREG 56
#endif
#define DORT_TRACE_REGS __maxnreg__(DORT_TRACE_MAXNREG)

template<class J>
__global__ void DORT_TRACE_REGS wf_extend(J jobs, WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  const uint32_t n = *(volatile uint32_t*)ctr_at(w.ctr, C_ACT0 + cur);
  const uint32_t* act = w.sorted ? w.sort_val[1] : w.active[cur];
  for(;;) {
    uint32_t base = warp_fetch(ctr_at(w.ctr, C_F_EXT));
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    uint32_t slot = 0, kind = kShadeQueues;
    if(i < n) {
      slot = act[i];
      uint32_t job = J::kBatched ? (w.meta[slot].w >> 8) : 0u;
      const PtScene& sc = jobs.scene(job);
      float4 o = w.ray_o[slot], d = w.ray_d[slot];
      Hit h = scene_trace<false, J::kGeneral>(sc, v3(o.x, o.y, o.z), o.w, v3(d.x, d.y, d.z),
                                              INFINITY);
      w.hit[slot] = make_float4(h.t, h.b1, h.b2, u2f(h.prim));
      kind = kMissQueue;
      if(h.prim != kMiss) {
        uint32_t mat = prim_material<J::kGeneral>(sc, h.prim);
        kind = __ldg(&sc.mats[mat].kind);
        // Oren-Nayar shares the Lambert queue (the queues only group work)
        if(kind >= kMissQueue) { kind = DORT_MAT_LAMBERT; }
      }
    }
    if(w.sorted) {
      if(i < n) { w.hit_kind[slot] = kind; }
      continue;
    }
#pragma unroll
    for(uint32_t k = 0; k < kShadeQueues; ++k) {
      bool mine = kind == k;
      uint32_t at = warp_append(ctr_at(w.ctr, C_KQ0 + k), mine);
      if(mine) { w.kq[k][at] = slot; }
    }
  }
}

// The direct lighting of one light at a path vertex (estimate_direct,
// path_renderer.cpp:135-206) as queue entries, `inv_lpdf` the inverse of the
// light's choice probability (1 when every light is sampled):
//   sh   the light strategy's shadow ray and its contribution if unblocked;
//   sh2  the BSDF strategy towards a background light: it counts only if the
//        ray escapes, and L and w depend on the direction alone, so it is an
//        any-hit query with its contribution computed here;
//   nb   the BSDF strategy towards an area light: closest hit, L and the MIS
//        weight once the hit is known (wf_neeb).
struct NeeEntries {
  bool sh, sh2, nb;
  float4 sh_o, sh_d, sh_c, sh2_o, sh2_d, sh2_c, nb_o, nb_d, nb_f;
};

template<bool G, bool ADJ = false>
__device__ __forceinline__ void nee_entries(const PtScene& sc, const PtParams& pp, uint32_t li,
                                            float inv_lpdf, const SurfaceHit& g,
                                            const DevMaterial& mt, V3 wo, V3 thr, float ub,
                                            float vb, float cb, float ul, float vl,
                                            NeeEntries& e) {
  const uint32_t req_nd = F_ALL & ~F_DELTA;
  e.sh = e.sh2 = e.nb = false;
  const DevLight& l = sc.lights[li];
  // the BSDF strategy only for area and background lights
  // (path_renderer.cpp:138-140)
  bool use_bsdf = pp.strategy != 2 && (light_is_area(l) || light_is_background(l));
  bool use_light = pp.strategy != 1;
  if(use_bsdf) {
    BsdfSample bs = bsdf_sample<G>(mt, g.frame, wo, req_nd, ub, vb, cb);
    if(!(bs.pdf == 0.f || is_black(bs.f))) {
      // contribution = f * L * (w |n.wi| / pdf) * thr / light_pick_pdf
      V3 fac = thr * (bs.f * (fabsf(dot(g.n, bs.w)) / bs.pdf)) * inv_lpdf;
      if(light_is_area(l)) {
        e.nb = true;
        e.nb_o = make_float4(g.p.x, g.p.y, g.p.z, g.eps);
        e.nb_d = make_float4(bs.w.x, bs.w.y, bs.w.z, bs.pdf);
        e.nb_f = make_float4(fac.x, fac.y, fac.z, u2f(li | (use_light ? 0x80000000u : 0u)));
      } else {
        V3 L = background_radiance(sc, l, bs.w);
        if(!is_black(L)) {
          float wgt = 1.f;
          if(use_light) {
            float lp = light_pivot_pdf<G>(sc, l, bs.w, g.p);
            wgt = bs.pdf / (bs.pdf + lp);
          }
          V3 c = fac * L * wgt;
          e.sh2 = true;
          e.sh2_o = make_float4(g.p.x, g.p.y, g.p.z, g.eps);
          e.sh2_d = make_float4(bs.w.x, bs.w.y, bs.w.z, INFINITY);
          e.sh2_c = make_float4(c.x, c.y, c.z, ADJ ? u2f(kMiss) : 0.f);
        }
      }
    }
  }
  if(use_light) {
    LightSample ls = light_sample<G>(sc, l, g.p, g.eps, ul, vl);
    if(!(ls.pdf == 0.f || is_black(ls.L))) {
      V3 f = bsdf_eval<G>(mt, g.frame, ls.wi, wo, req_nd);
      if(!is_black(f)) {
        float wgt = 1.f;
        if(use_bsdf) {
          float bp = bsdf_pdf<G>(mt, g.frame, ls.wi, wo, req_nd);
          wgt = ls.pdf / (ls.pdf + bp);
        }
        V3 c = (f * ls.L * (wgt * fabsf(dot(g.n, ls.wi)) / ls.pdf)) * inv_lpdf * thr;
        e.sh = true;
        e.sh_o = make_float4(ls.o.x, ls.o.y, ls.o.z, ls.tmin);
        e.sh_d = make_float4(ls.d.x, ls.d.y, ls.d.z, ls.tmax);
        // .w: for the adjoint, the light's triangle (its emission gradient)
        e.sh_c = make_float4(c.x, c.y, c.z,
                             ADJ ? u2f(l.kind == LIGHT_TRI ? l.tri : kMiss) : 0.f);
      }
    }
  }
}

// Appends one vertex's entries with per-thread atomics (the every-light mode,
// where a path adds a variable number of entries per wave).
__device__ __forceinline__ void push_entries(WfDev& w, uint32_t slot, const NeeEntries& e) {
  if(e.sh) {
    uint32_t at = atomicAdd(ctr_at(w.ctr, C_SHADOW), 1u);
    w.sh_slot[at] = slot; w.sh_o[at] = e.sh_o; w.sh_d[at] = e.sh_d; w.sh_c[at] = e.sh_c;
  }
  if(e.sh2) {
    uint32_t at = atomicAdd(ctr_at(w.ctr, C_SHADOW), 1u);
    w.sh_slot[at] = slot; w.sh_o[at] = e.sh2_o; w.sh_d[at] = e.sh2_d; w.sh_c[at] = e.sh2_c;
  }
  if(e.nb) {
    uint32_t at = atomicAdd(ctr_at(w.ctr, C_NEEB), 1u);
    w.nb_slot[at] = slot; w.nb_o[at] = e.nb_o; w.nb_d[at] = e.nb_d; w.nb_f[at] = e.nb_f;
  }
}

#ifdef DORT_SHADE_MAXNREG
#define DORT_SHADE_REGS __maxnreg__(DORT_SHADE_MAXNREG)
#else
#define DORT_SHADE_REGS
#endif

template<class J>
__global__ void DORT_SHADE_REGS wf_shade(J jobs, WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  uint32_t qn[kShadeQueues];
  uint32_t n = 0;
#pragma unroll
  for(uint32_t k = 0; k < kShadeQueues; ++k) {
    qn[k] = *(volatile uint32_t*)ctr_at(w.ctr, C_KQ0 + k);
    n += qn[k];
  }
  const uint32_t req_nd = F_ALL & ~F_DELTA;
  for(;;) {
    uint32_t base = warp_fetch(ctr_at(w.ctr, C_F_SHADE));
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    bool valid = i < n;
    bool cont = false, done = false;
    NeeEntries nee;
    nee.sh = nee.sh2 = nee.nb = false;
    uint32_t slot = 0;
    if(valid) {
      // index i of the concatenated shade queues
      uint32_t k = 0, off = i;
#pragma unroll
      for(uint32_t q = 0; q + 1 < kShadeQueues; ++q) {
        if(k == q && off >= qn[q]) { off -= qn[q]; k = q + 1; }
      }
      slot = w.kq[k][off];
      float4 ro = w.ray_o[slot], rd = w.ray_d[slot];
      float4 t4 = w.thr[slot], s4 = w.sum[slot];
      uint4 m = w.meta[slot];
      const uint32_t job = m.w >> 8;
      const PtScene& sc = jobs.scene(job);
      const PtParams& pp = jobs.params(job);
      float4 h4 = w.hit[slot];
      Hit h;
      h.t = h4.x; h.b1 = h4.y; h.b2 = h4.z; h.prim = f2u(h4.w);
      V3 o = v3(ro.x, ro.y, ro.z), d = v3(rd.x, rd.y, rd.z);
      V3 thr = v3(t4.x, t4.y, t4.z), sum = v3(s4.x, s4.y, s4.z);
      uint32_t bounces = m.z & kBounceMask;
      bool last_delta = (m.z >> 31) != 0;
      uint32_t next_oct = 0;
      bool hit = h.prim != kMiss;
      SurfaceHit g;
      if(hit) { g = surface_at<J::kGeneral>(sc, h, o, d); }
      if((bounces == 0 || last_delta) && bounces >= pp.min_depth && bounces <= pp.max_depth) {
        if(hit) {
          if(g.light) {
            const DevLight& l = sc.lights[g.light - 1];
            const V3 Le = area_eval_radiance(sc, l, g.p, g.n, o);
            if constexpr(J::kAdjoint) {
              if(jobs.d_emission && !is_black(Le) && g.tri < sc.shape_base) {
                adj_record<false>(w, slot, kEvEmission, g.tri, thr);
              }
            }
            sum = sum + thr * Le;
          }
        } else {
          for(uint32_t k = 0; k < sc.bg_count; ++k) {
            sum = sum + thr * background_radiance(sc, sc.lights[sc.bg_light[k]], d);
          }
        }
      }
      bounces += 1;
      bool finished = !hit || bounces > pp.max_depth;
      if(!finished) {
        V3 wo = normalize(-d);
        DevMaterial mt = material_at(sc, g);
        if constexpr(J::kAdjoint) {
          // a Lambert vertex: the sum of the terms so far and its albedo
          if(jobs.d_albedo && adj_albedo_vertex(mt, g.tri, sc.shape_base)) {
            const uint32_t k = adj_reserve<false>(w, slot, 2u);
            if(k + 2u <= kAdjLog) {
              w.adj_log[size_t(k) * w.capacity + slot] = adj_entry(kEvVertex, g.tri, sum);
              w.adj_log[size_t(k + 1u) * w.capacity + slot] =
                  adj_entry(kEvVertex, g.tri, v3(mt.c[0], mt.c[1], mt.c[2]));
            }
          }
        }
        uint32_t blk = bounce_block(bounces);
        Rand4 r0 = rand4(pp.seed, m.x, m.y, blk);
        Rand4 r1 = rand4(pp.seed, m.x, m.y, blk + 1);
        Rand4 r2 = rand4(pp.seed, m.x, m.y, blk + 2);
        if(bounces >= pp.min_depth && bxdf_matches(mt.bxdf_flags, req_nd) && sc.light_count > 0) {
          if(J::kGeneral && pp.sample_all_lights) {
            // every light, with its own random numbers (path_renderer.cpp:
            // 120-126); entries are appended one by one (this mode is for
            // scenes with few lights)
            for(uint32_t li = 0; li < sc.light_count; ++li) {
              uint32_t b2 = all_lights_block(bounces, li, sc.light_count);
              Rand4 a = rand4(pp.seed, m.x, m.y, b2);
              Rand4 b = rand4(pp.seed, m.x, m.y, b2 + 1);
              NeeEntries e;
              nee_entries<J::kGeneral, J::kAdjoint>(sc, pp, li, 1.f, g, mt, wo, thr, a.a, a.b,
                                                    a.c, b.a, b.b, e);
              push_entries(w, slot, e);
            }
          } else {
            uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, r0.a);
            float lpdf = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
            if(lpdf != 0.f) {
              nee_entries<J::kGeneral, J::kAdjoint>(sc, pp, li, 1.f / lpdf, g, mt, wo, thr, r0.b,
                                                    r0.c, r0.d, r1.a, r1.b, nee);
            }
          }
        }
        uint32_t req = (pp.only_direct || bounces == pp.max_depth) ? (F_MODES | F_DELTA) : F_ALL;
        BsdfSample bs = bsdf_sample<J::kGeneral>(mt, g.frame, wo, req, r1.c, r1.d, r2.a);
        if(is_black(bs.f) || bs.pdf == 0.f) {
          finished = true;
        } else {
          V3 contrib = bs.f * (fabsf(dot(bs.w, g.n)) / bs.pdf);
          last_delta = (bs.flags & F_DELTA) != 0;
          thr = thr * contrib;
          if(bounces == pp.max_depth && !last_delta) {
            finished = true;
          } else if(bounces >= 2 && bounces > pp.min_depth && pp.roulette) {
            float survive = clampf(average(contrib), 0.1f, 0.99f);
            if(r2.b > survive) {
              finished = true;
            } else {
              thr = thr * (1.f / survive);
            }
          }
          if(!finished) {
            w.ray_o[slot] = make_float4(g.p.x, g.p.y, g.p.z, g.eps);
            w.ray_d[slot] = make_float4(bs.w.x, bs.w.y, bs.w.z, 0.f);
            w.thr[slot] = make_float4(thr.x, thr.y, thr.z, 0.f);
            next_oct = dir_octant(bs.w);
          }
        }
      }
      w.sum[slot] = make_float4(sum.x, sum.y, sum.z, 0.f);
      m.z = bounces | (next_oct << kOctShift) | (last_delta ? 0x80000000u : 0u);
      m.w = (finished ? SLOT_FINISHED : SLOT_ACTIVE) | (job << 8);
      w.meta[slot] = m;
      cont = !finished;
      done = finished;
    }
    (void)cont;
    (void)done;
    uint32_t si = warp_append(ctr_at(w.ctr, C_SHADOW), nee.sh);
    if(nee.sh) {
      w.sh_slot[si] = slot;
      w.sh_o[si] = nee.sh_o;
      w.sh_d[si] = nee.sh_d;
      w.sh_c[si] = nee.sh_c;
    }
    uint32_t si2 = warp_append(ctr_at(w.ctr, C_SHADOW), nee.sh2);
    if(nee.sh2) {
      w.sh_slot[si2] = slot;
      w.sh_o[si2] = nee.sh2_o;
      w.sh_d[si2] = nee.sh2_d;
      w.sh_c[si2] = nee.sh2_c;
    }
    uint32_t ni = warp_append(ctr_at(w.ctr, C_NEEB), nee.nb);
    if(nee.nb) {
      w.nb_slot[ni] = slot;
      w.nb_o[ni] = nee.nb_o;
      w.nb_d[ni] = nee.nb_d;
      w.nb_f[ni] = nee.nb_f;
    }
  }
}

// One shadow-queue entry: any hit of its segment; if nothing blocks it, its
// contribution joins its path's sum.
template<class J>
__device__ __forceinline__ void shadow_entry(J& jobs, WfDev& w, uint32_t i, float4 o, float4 d) {
  uint32_t slot = w.sh_slot[i];
  uint32_t job = J::kBatched ? (w.meta[slot].w >> 8) : 0u;
  const PtScene& sc = jobs.scene(job);
  Hit h = scene_trace<true, J::kGeneral>(sc, v3(o.x, o.y, o.z), o.w, v3(d.x, d.y, d.z), d.w);
  if(h.prim == kMiss) {
    // a path can own two entries (light and BSDF strategy for a background
    // light), so the additions are atomic
    float4 c = w.sh_c[i];
    float* sp = &w.sum[slot].x;
    atomicAdd(sp, c.x);
    atomicAdd(sp + 1, c.y);
    atomicAdd(sp + 2, c.z);
    if constexpr(J::kAdjoint) {
      const uint32_t light_tri = f2u(c.w);
      if(jobs.d_emission && light_tri != kMiss) {
        adj_record<true>(w, slot, kEvDirect, light_tri, v3(c.x, c.y, c.z));
      }
    }
  }
}

// Staging of the shadow queue through the bulk-copy (TMA) engine.  The queue
// is contiguous in entry order, so a warp's next 32 entries (origins and
// directions, 512 bytes each) are one cp.async.bulk copy per array into the
// warp's slot of shared memory, completing on the warp's mbarrier; the warp
// issues the copy of its next batch as soon as it has read the current one
// into registers, so the loads of batch k + 1 overlap the traversals of
// batch k.  The source is this GPU's own memory and no copy multicasts.
constexpr uint32_t kTmaWarps = 8;   // blocks of up to 256 threads stage
constexpr uint32_t kTmaSpin = 1u << 20;   // bound on one mbarrier wait

struct ShadowStage {
  float4 o[32];
  float4 d[32];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return uint32_t(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// lane 0: arm the barrier for `bytes` and start the two copies into `st`
__device__ __forceinline__ void stage_batch(ShadowStage* st, uint64_t* bar, const float4* o,
                                            const float4* d, uint32_t count) {
  const uint32_t bytes = count * uint32_t(sizeof(float4));
  // the warp's earlier reads of the buffer (generic proxy) before the copy
  // (async proxy) overwrites it
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               ::"r"(smem_addr(bar)), "r"(2 * bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
               "[%0], [%1], %2, [%3];"
               ::"r"(smem_addr(st->o)), "l"(o), "r"(bytes), "r"(smem_addr(bar)) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
               "[%0], [%1], %2, [%3];"
               ::"r"(smem_addr(st->d)), "l"(d), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Bounded wait for the barrier's phase `parity`; warp-uniform result.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t spins) {
  uint32_t done = 0;
  for(uint32_t k = 0; k < spins && !done; ++k) {
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
                 "selp.u32 %0, 1, 0, p; }"
                 : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
  }
  return __any_sync(0xffffffffu, done != 0);
}

template<class J, bool STAGED>
__global__ void DORT_TRACE_REGS wf_shadow(J jobs, WfDev w) {
  const uint32_t n = *(volatile uint32_t*)ctr_at(w.ctr, C_SHADOW);
  const uint32_t lane = threadIdx.x & 31u;
  if(STAGED && blockDim.x <= 32 * kTmaWarps) {
    __shared__ __align__(128) ShadowStage stage[kTmaWarps];
    __shared__ __align__(8) uint64_t bar[kTmaWarps];
    const uint32_t warp = threadIdx.x >> 5;
    ShadowStage* st = &stage[warp];
    if(lane == 0) { mbar_init(&bar[warp]); }
    __syncwarp();
    uint32_t parity = 0;
    uint32_t base = warp_fetch(ctr_at(w.ctr, C_F_SH));
    if(base < n && lane == 0) {
      stage_batch(st, &bar[warp], w.sh_o + base, w.sh_d + base, min(32u, n - base));
    }
    while(base < n) {
      if(!mbar_wait(&bar[warp], parity, kTmaSpin)) {
        // the copy did not land: flag the frame (the host reports
        // DORT_ERR_TIMEOUT), wait longer for the copy in flight, stop
        if(lane == 0) { atomicOr(ctr_at(w.ctr, C_ERROR), 2u); }
        mbar_wait(&bar[warp], parity, 64u * kTmaSpin);
        return;
      }
      parity ^= 1u;
      const uint32_t i = base + lane;
      float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = o;
      if(i < n) {
        o = st->o[lane];
        d = st->d[lane];
      }
      __syncwarp();
      const uint32_t next = warp_fetch(ctr_at(w.ctr, C_F_SH));
      if(next < n && lane == 0) {
        stage_batch(st, &bar[warp], w.sh_o + next, w.sh_d + next, min(32u, n - next));
      }
      if(i < n) { shadow_entry(jobs, w, i, o, d); }
      base = next;
    }
    return;
  }
  for(;;) {
    uint32_t base = warp_fetch(ctr_at(w.ctr, C_F_SH));
    if(base >= n) { break; }
    uint32_t i = base + lane;
    if(i < n) { shadow_entry(jobs, w, i, w.sh_o[i], w.sh_d[i]); }
  }
}

template<bool G, bool ADJ>
__device__ __forceinline__ void neeb_one_impl(const PtScene& sc, WfDev& w, uint32_t i,
                                              bool want_emission);

template<class J>
__global__ void wf_neeb(J jobs, WfDev w) {
  const uint32_t n = *(volatile uint32_t*)ctr_at(w.ctr, C_NEEB);
  for(;;) {
    uint32_t base = warp_fetch(ctr_at(w.ctr, C_F_NB));
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    if(i < n) {
      uint32_t job = J::kBatched ? (w.meta[w.nb_slot[i]].w >> 8) : 0u;
      bool want_emission = false;
      if constexpr(J::kAdjoint) { want_emission = jobs.d_emission != nullptr; }
      neeb_one_impl<J::kGeneral, J::kAdjoint>(jobs.scene(job), w, i, want_emission);
    }
  }
}

template<bool G, bool ADJ>
__device__ __forceinline__ void neeb_one_impl(const PtScene& sc, WfDev& w, uint32_t i,
                                              bool want_emission) {
    float4 o = w.nb_o[i], d = w.nb_d[i], f = w.nb_f[i];
    uint32_t lw = f2u(f.w);
    const uint32_t li = lw & 0x7fffffffu;
    const DevLight& l = sc.lights[li];
    bool use_mis = (lw >> 31) != 0;
    V3 L = v3(0.f, 0.f, 0.f);
    V3 p = v3(o.x, o.y, o.z), wi = v3(d.x, d.y, d.z);
    if(light_is_area(l)) {
      Hit h = scene_trace<false, G>(sc, p, o.w, wi, INFINITY);
      L = area_light_hit_radiance<G>(sc, li, h, p, wi);
    } else {
      // background light: only escaping rays count, an any-hit query decides
      Hit h = scene_trace<true, G>(sc, p, o.w, wi, INFINITY);
      if(h.prim == kMiss) { L = background_radiance(sc, l, wi); }
    }
    if(!is_black(L)) {
      float wgt = 1.f;
      if(use_mis) {
        float lp = light_pivot_pdf<G>(sc, l, wi, p);
        wgt = d.w / (d.w + lp);
      }
      V3 c = v3(f.x, f.y, f.z) * L * wgt;
      // with sample_all_lights a path owns one entry per area light, which
      // may run in the same wave of this kernel: the additions are atomic
      float* sp = &w.sum[w.nb_slot[i]].x;
      atomicAdd(sp, c.x);
      atomicAdd(sp + 1, c.y);
      atomicAdd(sp + 2, c.z);
      if(ADJ && want_emission && l.kind == LIGHT_TRI) {
        adj_record<true>(w, w.nb_slot[i], kEvDirect, l.tri, c);
      }
    }
}

// Single thread: account the wave, retire its queues, decide whether to loop.
__device__ __forceinline__ bool wf_end_wave(WfDev& w) {
  uint32_t wave = *ctr_at(w.ctr, C_WAVES);
  uint32_t cur = wave & 1u;
  uint32_t a = *ctr_at(w.ctr, C_ACT0 + cur), s = *ctr_at(w.ctr, C_SHADOW), b = *ctr_at(w.ctr, C_NEEB);
  unsigned long long* rays = reinterpret_cast<unsigned long long*>(ctr_at(w.ctr, C_RAYS_LO));
  *rays += (unsigned long long)a + s + b;
  // this wave's active queue stays for the next regen; the lists this wave's
  // regen read are consumed
  *ctr_at(w.ctr, C_ACT0 + (cur ^ 1u)) = 0u;
  *ctr_at(w.ctr, C_FIN0 + cur) = 0u;
  *ctr_at(w.ctr, C_SHADOW) = 0u;
  *ctr_at(w.ctr, C_NEEB) = 0u;
  *ctr_at(w.ctr, C_F_EXT) = 0u;
  *ctr_at(w.ctr, C_F_SHADE) = 0u;
  *ctr_at(w.ctr, C_F_SH) = 0u;
  *ctr_at(w.ctr, C_F_NB) = 0u;
  for(uint32_t k = 0; k < kShadeQueues; ++k) { *ctr_at(w.ctr, C_KQ0 + k) = 0u; }
  *ctr_at(w.ctr, C_WAVES) = wave + 1u;
  uint64_t next = *reinterpret_cast<uint64_t*>(ctr_at(w.ctr, C_NEXT_LO));
  bool more = *ctr_at(w.ctr, C_LIVE) > 0u || next < w.total_samples;
  if(more && wave + 1u >= w.max_waves) {
    // bounded: a frame never loops forever; the host reports the error
    *ctr_at(w.ctr, C_ERROR) = 1u;
    more = false;
  }
  return more;
}

__global__ void wf_control(WfDev w, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, wf_end_wave(w) ? 1u : 0u);
}

__global__ void wf_resolve(WfDev w, uint32_t npix, float* __restrict__ out) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if(p < npix) {
    float4 a = w.film[p];
    float inv = a.w != 0.f ? 1.f / a.w : 0.f;
    out[3 * size_t(p)] = a.w != 0.f ? a.x * inv : 0.f;
    out[3 * size_t(p) + 1] = a.w != 0.f ? a.y * inv : 0.f;
    out[3 * size_t(p) + 2] = a.w != 0.f ? a.z * inv : 0.f;
  }
}

// The deterministic resolve: every pixel's unit sums in unit order.
__global__ void wf_resolve_units(WfDev w, uint32_t npix, uint32_t units,
                                 float* __restrict__ out) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if(p >= npix) { return; }
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
  for(uint32_t u = 0; u < units; ++u) {
    const float4 b = w.unit_film[size_t(u) * npix + p];
    a = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
  }
  const float inv = a.w != 0.f ? 1.f / a.w : 0.f;
  out[3 * size_t(p)] = a.x * inv;
  out[3 * size_t(p) + 1] = a.y * inv;
  out[3 * size_t(p) + 2] = a.z * inv;
}

// ---- host side --------------------------------------------------------------------

struct Wavefront {
  WfDev dev{};
  cudaStream_t capture_stream = nullptr;   // graphs cannot be captured on stream 0
  void* mem = nullptr;
  size_t mem_bytes = 0;
  uint32_t capacity = 0;
  uint32_t npix_cap = 0;
  uint32_t nee_mult = 1;
  // graph cache (rebuilt when parameters change)
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  PtParams pp_cached{};
  PtScene sc_cached{};     // the scene view the graph's kernels were given
  const void* jobs_cached = nullptr;
  WfTuning tune_cached{};
  bool valid = false;
  // per-unit sums of deterministic frames (grow-only)
  void* unit_mem = nullptr;
  size_t unit_bytes = 0;
  // the adjoint's term log (allocated by the adjoint's backward pass only)
  void* adj_mem = nullptr;
  uint32_t adj_capacity = 0;
  uint64_t adj_key[6] = {0, 0, 0, 0, 0, 0};   // the adjoint buffers the graph was given
};

static void wf_release(Wavefront* wf) {
  if(wf->capture_stream) { cudaStreamDestroy(wf->capture_stream); wf->capture_stream = nullptr; }
  if(wf->exec) { cudaGraphExecDestroy(wf->exec); wf->exec = nullptr; }
  if(wf->graph) { cudaGraphDestroy(wf->graph); wf->graph = nullptr; }
  if(wf->mem) { cudaFree(wf->mem); wf->mem = nullptr; }
  if(wf->adj_mem) { cudaFree(wf->adj_mem); wf->adj_mem = nullptr; }
  wf->adj_capacity = 0;
  if(wf->unit_mem) { cudaFree(wf->unit_mem); wf->unit_mem = nullptr; }
  wf->unit_bytes = 0;
  wf->dev.unit_film = nullptr;
  wf->dev.adj_log = nullptr;
  wf->dev.adj_n = nullptr;
  wf->valid = false;
}

void wavefront_destroy(Wavefront* wf) {
  if(!wf) { return; }
  wf_release(wf);
  delete wf;
}

// Entries a path adds to the direct-lighting queues per wave, relative to
// one light: every light when the frame samples them all.
static uint32_t nee_mult(const PtScene& sc, const PtParams& pp) {
  return pp.sample_all_lights ? std::max(1u, sc.light_count) : 1u;
}

// Queues of `capacity` path slots for images of up to npix pixels; a path
// adds up to 2 * nee_mult shadow entries and nee_mult BSDF-strategy entries
// per wave (nee_mult = the light count when every light is sampled, else 1).
static int wf_alloc(Wavefront* wf, uint32_t capacity, uint32_t npix, uint32_t nee_mult = 1) {
  if(wf->mem && wf->capacity == capacity && wf->npix_cap >= npix && wf->nee_mult == nee_mult) {
    return DORT_OK;
  }
  // the direct-lighting queues' entries are counted in 32 bits
  if(!wavefront_entries_fit(capacity, nee_mult)) {
    return fail(DORT_ERR_INVALID, "queue_capacity x sampled lights too large: " +
                std::to_string(capacity) + " path slots x " + std::to_string(nee_mult) +
                " lights exceeds 2^30 direct-lighting entries per wave");
  }
  wf_release(wf);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t Q = capacity;
  size_t f4 = al(Q * sizeof(float4)), u4 = al(Q * sizeof(uint4)), u1 = al(Q * sizeof(uint32_t));
  size_t f4x2 = al(2 * nee_mult * Q * sizeof(float4));
  size_t u1x2 = al(2 * nee_mult * Q * sizeof(uint32_t));
  size_t f4n = al(nee_mult * Q * sizeof(float4)), u1n = al(nee_mult * Q * sizeof(uint32_t));
  size_t sort_temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_temp, static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), int(capacity), 0, kSortBits);
  sort_temp = al(sort_temp);
  size_t bytes = 5 * f4 + u4 + f4 /*hit*/ + (4 + kShadeQueues) * u1 /*queues*/ + u1x2 +
                 3 * f4x2 /*shadow, two per path*/ + u1n + 3 * f4n /*neeb*/ +
                 al(size_t(npix) * sizeof(float4)) + 5 * u1 /*sort*/ + sort_temp +
                 al(C_COUNT * kCtrStride * 4);
  if(dev_alloc(&wf->mem, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(DORT_ERR_OOM, "cudaMalloc of wavefront queues failed (" +
                std::to_string(bytes) + " bytes)");
  }
  char* p = static_cast<char*>(wf->mem);
  auto take = [&](size_t b) { char* r = p; p += b; return r; };
  WfDev& d = wf->dev;
  d.ray_o = reinterpret_cast<float4*>(take(f4));
  d.ray_d = reinterpret_cast<float4*>(take(f4));
  d.thr = reinterpret_cast<float4*>(take(f4));
  d.sum = reinterpret_cast<float4*>(take(f4));
  d.acc = reinterpret_cast<float4*>(take(f4));
  d.meta = reinterpret_cast<uint4*>(take(u4));
  d.hit = reinterpret_cast<float4*>(take(f4));
  d.active[0] = reinterpret_cast<uint32_t*>(take(u1));
  d.active[1] = reinterpret_cast<uint32_t*>(take(u1));
  d.finished[0] = reinterpret_cast<uint32_t*>(take(u1));
  d.finished[1] = reinterpret_cast<uint32_t*>(take(u1));
  for(uint32_t k = 0; k < kShadeQueues; ++k) { d.kq[k] = reinterpret_cast<uint32_t*>(take(u1)); }
  d.sh_slot = reinterpret_cast<uint32_t*>(take(u1x2));
  d.sh_o = reinterpret_cast<float4*>(take(f4x2));
  d.sh_d = reinterpret_cast<float4*>(take(f4x2));
  d.sh_c = reinterpret_cast<float4*>(take(f4x2));
  d.nb_slot = reinterpret_cast<uint32_t*>(take(u1n));
  d.nb_o = reinterpret_cast<float4*>(take(f4n));
  d.nb_d = reinterpret_cast<float4*>(take(f4n));
  d.nb_f = reinterpret_cast<float4*>(take(f4n));
  d.film = reinterpret_cast<float4*>(take(al(size_t(npix) * sizeof(float4))));
  for(int k = 0; k < 2; ++k) {
    d.sort_key[k] = reinterpret_cast<uint32_t*>(take(u1));
    d.sort_val[k] = reinterpret_cast<uint32_t*>(take(u1));
  }
  d.hit_kind = reinterpret_cast<uint32_t*>(take(u1));
  d.sort_temp = take(sort_temp);
  d.sort_temp_bytes = sort_temp;
  d.ctr = reinterpret_cast<uint32_t*>(take(al(C_COUNT * kCtrStride * 4)));
  d.capacity = capacity;
  wf->capacity = capacity;
  wf->npix_cap = npix;
  wf->nee_mult = nee_mult;
  wf->mem_bytes = bytes;
  return DORT_OK;
}

static int grid_for(const void* kernel, int block) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
  return sms * std::max(per_sm, 1);
}

// Grid and block of every stage kernel.  A block size the tuning asks for
// that a kernel's registers do not allow (threads x registers above the
// SM's register file) is lowered to the kernel's limit, a multiple of 32.
struct WfGrids {
  int regen, ext, sha, shw, nb;
  int b_ext, b_sha, b_shw, b_nb;
};

static int fit_block(const void* kernel, int block) {
  cudaFuncAttributes a{};
  if(cudaFuncGetAttributes(&a, kernel) != cudaSuccess) {
    cudaGetLastError();
    return block;
  }
  return std::min(block, std::max(32, a.maxThreadsPerBlock & ~31));
}

template<class J>
static WfGrids wf_grids(const WfTuning& tn) {
  WfGrids g;
  const void* ext = reinterpret_cast<const void*>(&wf_extend<J>);
  const void* sha = reinterpret_cast<const void*>(&wf_shade<J>);
  const void* shw = tn.stage_queues ? reinterpret_cast<const void*>(&wf_shadow<J, true>)
                                    : reinterpret_cast<const void*>(&wf_shadow<J, false>);
  const void* nb = reinterpret_cast<const void*>(&wf_neeb<J>);
  g.b_ext = fit_block(ext, int(tn.trace_block));
  g.b_sha = fit_block(sha, int(tn.shade_block));
  g.b_shw = fit_block(shw, int(tn.trace_block));
  g.b_nb = fit_block(nb, int(tn.trace_block));
  g.regen = grid_for(reinterpret_cast<const void*>(&wf_regen<J>), int(kRegenBlock));
  g.ext = grid_for(ext, g.b_ext);
  g.sha = grid_for(sha, g.b_sha);
  g.shw = grid_for(shw, g.b_shw);
  g.nb = grid_for(nb, g.b_nb);
  return g;
}

// The ray sort between regeneration and extension (tn.sort).
template<class J>
static void wf_sort(const J& jobs, WfDev& dev, const WfGrids& g, cudaStream_t st) {
  wf_sort_keys<J><<<g.regen, 256, 0, st>>>(jobs, dev);
  size_t tb = dev.sort_temp_bytes;
  cub::DeviceRadixSort::SortPairs(dev.sort_temp, tb, dev.sort_key[0], dev.sort_key[1],
                                  dev.sort_val[0], dev.sort_val[1], int(dev.capacity), 0,
                                  kSortBits, st);
}

// The extension stage (with the ray sort and the classification that go
// with it) and the shadow stage in the variants the tuning selects.
template<class J>
static void wf_launch_extend(const J& jobs, WfDev& dev, const WfTuning& tn, const WfGrids& g,
                             cudaStream_t st) {
  if(tn.sort) { wf_sort<J>(jobs, dev, g, st); }
  wf_extend<J><<<g.ext, g.b_ext, 0, st>>>(jobs, dev);
  if(tn.sort) { wf_classify<<<g.regen, 256, 0, st>>>(dev); }
}

template<class J>
static void wf_launch_shadow(const J& jobs, WfDev& dev, const WfTuning& tn, const WfGrids& g,
                             cudaStream_t st) {
  if(tn.stage_queues) {
    wf_shadow<J, true><<<g.shw, g.b_shw, 0, st>>>(jobs, dev);
  } else {
    wf_shadow<J, false><<<g.shw, g.b_shw, 0, st>>>(jobs, dev);
  }
}

template<class J>
static void wf_launch_wave(const J& jobs, WfDev& dev, const WfTuning& tn, const WfGrids& g,
                           cudaStream_t st) {
  wf_regen<J><<<g.regen, kRegenBlock, 0, st>>>(jobs, dev);
  wf_launch_extend<J>(jobs, dev, tn, g, st);
  wf_shade<J><<<g.sha, g.b_sha, 0, st>>>(jobs, dev);
  wf_launch_shadow<J>(jobs, dev, tn, g, st);
  wf_neeb<J><<<g.nb, g.b_nb, 0, st>>>(jobs, dev);
}

template<class J>
static int wf_build_graph(Wavefront* wf, const J& jobs, const WfTuning& tn) {
  if(!wf->capture_stream) {
    DG_CUDA(cudaStreamCreateWithFlags(&wf->capture_stream, cudaStreamNonBlocking));
  }
  cudaStream_t st = wf->capture_stream;
  if(wf->exec) { cudaGraphExecDestroy(wf->exec); wf->exec = nullptr; }
  if(wf->graph) { cudaGraphDestroy(wf->graph); wf->graph = nullptr; }
  wf->valid = false;
  DG_CUDA(cudaGraphCreate(&wf->graph, 0));
  cudaGraphConditionalHandle handle;
  DG_CUDA(cudaGraphConditionalHandleCreate(&handle, wf->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  DG_CUDA(cudaGraphAddNode(&cnode, wf->graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  WfGrids g = wf_grids<J>(tn);
  wf->dev.sorted = tn.sort;
  DG_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  wf_launch_wave<J>(jobs, wf->dev, tn, g, st);
  wf_control<<<1, 1, 0, st>>>(wf->dev, handle);
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(st, &captured);
  if(ce != cudaSuccess) {
    return fail(DORT_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(ce));
  }
  DG_CUDA(cudaGraphInstantiate(&wf->exec, wf->graph, 0));
  wf->tune_cached = tn;
  wf->valid = true;
  return DORT_OK;
}

static uint32_t wave_bound(uint64_t total_units, uint32_t capacity, uint32_t max_depth,
                           uint32_t cap = 0) {
  // each slot runs at most ceil(units / capacity) + 1 units of kChunk samples
  // of at most max_depth + 2 waves each; a caller's cap (tuning.max_waves)
  // may lower the bound
  uint64_t b = std::min<uint64_t>(
      0x7fffffffull, (total_units / std::max(1u, capacity) + 2) * kChunk *
                     (uint64_t(max_depth) + 3) + 64);
  if(cap) { b = std::min<uint64_t>(b, cap); }
  return uint32_t(b);
}

// Work units of a frame (kChunk samples of one pixel each, padded to whole
// 8x4 tiles).
static uint64_t padded_samples(const PtParams& pp) {
  uint64_t tiles = uint64_t((pp.width + 7) / 8) * ((pp.height + 3) / 4);
  return tiles * 32 * ((pp.spp + kChunk - 1) / kChunk);
}

int wavefront_render(dort_scene* s, const PtParams& pp, const WfTuning& tn, float* d_out,
                     cudaStream_t st) {
  if(!s->wavefront) { s->wavefront = new Wavefront(); }
  Wavefront* wf = s->wavefront;
  uint32_t npix = pp.width * pp.height;
  int rc = wf_alloc(wf, tn.capacity, npix, nee_mult(s->pt, pp));
  if(rc != DORT_OK) { return rc; }
  const uint32_t units = (pp.spp + kChunk - 1) / kChunk;
  float4* unit_film = nullptr;
  if(tn.deterministic) {
    const size_t need = size_t(npix) * units * sizeof(float4);
    if(wf->unit_bytes < need) {
      if(wf->unit_mem) { cudaFree(wf->unit_mem); }
      wf->unit_mem = nullptr;
      wf->unit_bytes = 0;
      if(dev_alloc(&wf->unit_mem, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(DORT_ERR_OOM, "cudaMalloc of the per-unit sums failed");
      }
      wf->unit_bytes = need;
    }
    unit_film = static_cast<float4*>(wf->unit_mem);
  }
  if(wf->dev.unit_film != unit_film || wf->dev.npix != npix) { wf->valid = false; }
  wf->dev.unit_film = unit_film;
  wf->dev.npix = npix;
  wf->dev.total_samples = padded_samples(pp);
  wf->dev.max_waves = wave_bound(wf->dev.total_samples, tn.capacity, pp.max_depth, tn.max_waves);
  // the graph holds the scene view by value: a change to it (per-triangle
  // parameters set or cleared by the adjoint entry points) rebuilds it
  if(!wf->valid || wf->jobs_cached != nullptr ||
     std::memcmp(&wf->pp_cached, &pp, sizeof(PtParams)) != 0 ||
     std::memcmp(&wf->sc_cached, &s->pt, sizeof(PtScene)) != 0 ||
     std::memcmp(&wf->tune_cached, &tn, sizeof(WfTuning)) != 0) {
    rc = scene_needs_general(s->pt, pp) ? wf_build_graph(wf, SingleJob<true>{s->pt, pp}, tn)
                                        : wf_build_graph(wf, SingleJob<false>{s->pt, pp}, tn);
    if(rc != DORT_OK) { return rc; }
    wf->pp_cached = pp;
    std::memcpy(&wf->sc_cached, &s->pt, sizeof(PtScene));
    wf->jobs_cached = nullptr;
  }
  // the graph holds the kernel arguments, including total_samples and max_waves
  wf_init<<<(std::max(tn.capacity, npix) + 255) / 256, 256, 0, st>>>(wf->dev, npix);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaGraphLaunch(wf->exec, st));
  if(unit_film) {
    wf_resolve_units<<<(npix + 255) / 256, 256, 0, st>>>(wf->dev, npix, units, d_out);
  } else {
    wf_resolve<<<(npix + 255) / 256, 256, 0, st>>>(wf->dev, npix, d_out);
  }
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

// The adjoint's backward pass (AdjointJob): one wavefront frame whose paths
// log their terms; the slot logs hold kAdjLog entries of 16 bytes per slot.
int wavefront_adjoint(dort_scene* s, const PtParams& pp, const WfTuning& tn, const float* d_dl,
                      float* d_ga, float* d_ge, uint2* d_overflow, uint32_t overflow_cap,
                      uint32_t* d_overflow_n, cudaStream_t st) {
  if(!s->adj_wavefront) { s->adj_wavefront = new Wavefront(); }
  Wavefront* wf = s->adj_wavefront;
  const uint32_t npix = pp.width * pp.height;
  int rc = wf_alloc(wf, tn.capacity, npix, nee_mult(s->pt, pp));
  if(rc != DORT_OK) { return rc; }
  if(!wf->adj_mem || wf->adj_capacity != tn.capacity) {
    if(wf->adj_mem) { cudaFree(wf->adj_mem); wf->adj_mem = nullptr; }
    const size_t log_bytes = size_t(kAdjLog) * tn.capacity * sizeof(float4);
    if(dev_alloc(&wf->adj_mem, log_bytes + size_t(tn.capacity) * sizeof(uint32_t)) !=
       cudaSuccess) {
      cudaGetLastError();
      wf->adj_capacity = 0;
      wf->dev.adj_log = nullptr;
      wf->dev.adj_n = nullptr;
      return fail(DORT_ERR_OOM, "cudaMalloc of the adjoint's term log failed");
    }
    wf->adj_capacity = tn.capacity;
    wf->dev.adj_log = static_cast<float4*>(wf->adj_mem);
    wf->dev.adj_n = reinterpret_cast<uint32_t*>(static_cast<char*>(wf->adj_mem) + log_bytes);
    wf->valid = false;
  }
  wf->dev.total_samples = padded_samples(pp);
  wf->dev.max_waves = wave_bound(wf->dev.total_samples, tn.capacity, pp.max_depth, tn.max_waves);
  const uint64_t key[6] = {uint64_t(uintptr_t(d_dl)), uint64_t(uintptr_t(d_ga)),
                           uint64_t(uintptr_t(d_ge)), uint64_t(uintptr_t(d_overflow)),
                           uint64_t(uintptr_t(d_overflow_n)), overflow_cap};
  if(!wf->valid || std::memcmp(&wf->pp_cached, &pp, sizeof(PtParams)) != 0 ||
     std::memcmp(&wf->sc_cached, &s->pt, sizeof(PtScene)) != 0 ||
     std::memcmp(&wf->tune_cached, &tn, sizeof(WfTuning)) != 0 ||
     std::memcmp(wf->adj_key, key, sizeof(key)) != 0) {
    auto build = [&](auto job) {
      job.sc = s->pt;
      job.pp = pp;
      job.dl_dimage = d_dl;
      job.d_albedo = d_ga;
      job.d_emission = d_ge;
      job.overflow = d_overflow;
      job.overflow_n = d_overflow_n;
      job.overflow_cap = overflow_cap;
      return wf_build_graph(wf, job, tn);
    };
    rc = scene_needs_general(s->pt, pp) ? build(AdjointJob<true>{}) : build(AdjointJob<false>{});
    if(rc != DORT_OK) { return rc; }
    wf->pp_cached = pp;
    std::memcpy(&wf->sc_cached, &s->pt, sizeof(PtScene));
    std::memcpy(wf->adj_key, key, sizeof(key));
    wf->jobs_cached = nullptr;
  }
  wf_init<<<(std::max(tn.capacity, npix) + 255) / 256, 256, 0, st>>>(wf->dev, npix);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaGraphLaunch(wf->exec, st));
  return DORT_OK;
}

int wavefront_counters_of(Wavefront* wf, uint64_t* rays, uint32_t* waves, uint32_t* error,
                          cudaStream_t st);

int wavefront_adjoint_counters(dort_scene* s, uint64_t* rays, uint32_t* waves, uint32_t* error,
                               cudaStream_t st) {
  return wavefront_counters_of(s->adj_wavefront, rays, waves, error, st);
}

// The same frame as wavefront_render, run wave by wave from the host without
// the graph, with CUDA events around every stage; for measurement only.
__global__ void wf_control_host(WfDev w, uint32_t* more_flag) {
  *more_flag = wf_end_wave(w) ? 1u : 0u;
}

template<bool G>
static int stage_times_g(dort_scene* s, const PtParams& pp, const WfTuning& tn, float* d_out,
                         cudaStream_t st, double ms[6], double stage_rays[3]) {
  if(!s->wavefront) { s->wavefront = new Wavefront(); }
  Wavefront* wf = s->wavefront;
  uint32_t npix = pp.width * pp.height;
  int rc = wf_alloc(wf, tn.capacity, npix, nee_mult(s->pt, pp));
  if(rc != DORT_OK) { return rc; }
  // film sums by atomics here (wf_resolve); the cached graph is rebuilt by
  // the next frame that wants per-unit sums
  if(wf->dev.unit_film) {
    wf->dev.unit_film = nullptr;
    wf->valid = false;
  }
  wf->dev.npix = npix;
  wf->dev.total_samples = padded_samples(pp);
  wf->dev.max_waves = wave_bound(wf->dev.total_samples, tn.capacity, pp.max_depth, tn.max_waves);
  SingleJob<G> jobs{s->pt, pp};
  WfGrids g = wf_grids<SingleJob<G>>(tn);
  wf->dev.sorted = tn.sort;
  // more[0]: loop flag; more[1..6]: the counters C_ACT0 .. C_NEEB of the wave
  uint32_t* more = nullptr;
  DG_CUDA(host_pinned_alloc(&more, 8 * sizeof(uint32_t)));
  cudaEvent_t ev[6];
  for(auto& e : ev) { cudaEventCreate(&e); }
  for(int k = 0; k < 6; ++k) { ms[k] = 0.0; }
  for(int k = 0; k < 3; ++k) { stage_rays[k] = 0.0; }
  wf_init<<<(std::max(tn.capacity, npix) + 255) / 256, 256, 0, st>>>(wf->dev, npix);
  bool ok = cudaGetLastError() == cudaSuccess;
  for(uint32_t wave = 0; ok && wave < wf->dev.max_waves + 1; ++wave) {
    cudaEventRecord(ev[0], st);
    wf_regen<SingleJob<G>><<<g.regen, kRegenBlock, 0, st>>>(jobs, wf->dev);
    cudaEventRecord(ev[1], st);
    // the sort counts as part of the extension stage
    wf_launch_extend<SingleJob<G>>(jobs, wf->dev, tn, g, st);
    cudaEventRecord(ev[2], st);
    wf_shade<SingleJob<G>><<<g.sha, g.b_sha, 0, st>>>(jobs, wf->dev);
    cudaEventRecord(ev[3], st);
    wf_launch_shadow<SingleJob<G>>(jobs, wf->dev, tn, g, st);
    cudaEventRecord(ev[4], st);
    wf_neeb<SingleJob<G>><<<g.nb, g.b_nb, 0, st>>>(jobs, wf->dev);
    cudaEventRecord(ev[5], st);
    cudaMemcpy2DAsync(more + 1, sizeof(uint32_t), wf->dev.ctr, kCtrStride * sizeof(uint32_t),
                      sizeof(uint32_t), C_NEEB + 1, cudaMemcpyDeviceToHost, st);
    wf_control_host<<<1, 1, 0, st>>>(wf->dev, more);
    ok = cudaStreamSynchronize(st) == cudaSuccess;
    for(int k = 0; ok && k < 5; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      ms[k] += t;
    }
    if(ok) {
      stage_rays[0] += double(more[1 + C_ACT0 + (wave & 1u)]);
      stage_rays[1] += double(more[1 + C_SHADOW]);
      stage_rays[2] += double(more[1 + C_NEEB]);
    }
    if(!*more) { break; }
  }
  if(ok) {
    wf_resolve<<<(npix + 255) / 256, 256, 0, st>>>(wf->dev, npix, d_out);
    ok = cudaStreamSynchronize(st) == cudaSuccess;
  }
  for(auto& e : ev) { cudaEventDestroy(e); }
  cudaFreeHost(more);
  ms[5] = 0.0;
  // the graph cache no longer matches the queues' state; rebuild next time
  wf->valid = false;
  if(!ok) {
    return fail(DORT_ERR_CUDA, std::string("staged wavefront failed: ") +
                               cudaGetErrorString(cudaGetLastError()));
  }
  return DORT_OK;
}

int wavefront_stage_times(dort_scene* s, const PtParams& pp, const WfTuning& tn,
                          float* d_out, cudaStream_t st, double ms[6], double stage_rays[3]) {
  return scene_needs_general(s->pt, pp)
      ? stage_times_g<true>(s, pp, tn, d_out, st, ms, stage_rays)
      : stage_times_g<false>(s, pp, tn, d_out, st, ms, stage_rays);
}

int wavefront_counters_of(Wavefront* wf, uint64_t* rays, uint32_t* waves, uint32_t* error,
                          cudaStream_t st) {
  if(!wf || !wf->mem) { return fail(DORT_ERR_INVALID, "no wavefront state"); }
  // the first two words of every counter's line
  uint32_t c[2 * C_COUNT];
  DG_CUDA(cudaMemcpy2DAsync(c, 2 * sizeof(uint32_t), wf->dev.ctr, kCtrStride * sizeof(uint32_t),
                            2 * sizeof(uint32_t), C_COUNT, cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaStreamSynchronize(st));
  *rays = uint64_t(c[2 * C_RAYS_LO]) | (uint64_t(c[2 * C_RAYS_LO + 1]) << 32);
  *waves = c[2 * C_WAVES];
  *error = c[2 * C_ERROR];
  return DORT_OK;
}

int wavefront_counters(dort_scene* s, uint64_t* rays, uint32_t* waves, uint32_t* error,
                       cudaStream_t st) {
  return wavefront_counters_of(s->wavefront, rays, waves, error, st);
}

// ---- batches of frames ------------------------------------------------------------

__global__ void wf_resolve_batch(WfDev w, const WfJob* jobs, uint32_t job_count,
                                 uint32_t total_pix, float* __restrict__ out) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if(p >= total_pix) { return; }
  float4 a = w.film[p];
  float inv = a.w != 0.f ? 1.f / a.w : 0.f;
  out[3 * size_t(p)] = a.w != 0.f ? a.x * inv : 0.f;
  out[3 * size_t(p) + 1] = a.w != 0.f ? a.y * inv : 0.f;
  out[3 * size_t(p) + 2] = a.w != 0.f ? a.z * inv : 0.f;
  (void)jobs;
  (void)job_count;
}

struct WavefrontBatch {
  Wavefront wf;
  WfJob* d_jobs = nullptr;
  float* d_images = nullptr;
  uint32_t job_count = 0;
  uint32_t total_pix = 0;
  uint64_t total_samples = 0;
  uint32_t max_depth = 0;
  uint32_t nee_mult = 1;
  WfTuning tn{};
  std::vector<uint32_t> film_offset;
  std::vector<uint32_t> npix;
};

void wavefront_batch_destroy(WavefrontBatch* b) {
  if(!b) { return; }
  wf_release(&b->wf);
  if(b->d_jobs) { cudaFree(b->d_jobs); }
  if(b->d_images) { cudaFree(b->d_images); }
  delete b;
}

int wavefront_batch_create(const PtScene* scenes, const PtParams* params, uint32_t n,
                           const WfTuning& tn, WavefrontBatch** out) {
  auto* b = new WavefrontBatch();
  std::vector<WfJob> jobs(n);
  uint64_t sample = 0;
  uint32_t pix = 0;
  for(uint32_t j = 0; j < n; ++j) {
    std::memset(&jobs[j], 0, sizeof(WfJob));
    jobs[j].sc = scenes[j];
    jobs[j].pp = params[j];
    jobs[j].sample_begin = sample;
    jobs[j].film_offset = pix;
    b->film_offset.push_back(pix);
    b->npix.push_back(params[j].width * params[j].height);
    sample += padded_samples(params[j]);
    uint64_t np = uint64_t(pix) + uint64_t(params[j].width) * params[j].height;
    if(np > 0x7fffffffull) {
      delete b;
      return fail(DORT_ERR_INVALID, "batch exceeds 2^31 pixels");
    }
    pix = uint32_t(np);
    b->max_depth = std::max(b->max_depth, params[j].max_depth);
    b->nee_mult = std::max(b->nee_mult, nee_mult(scenes[j], params[j]));
  }
  b->job_count = n;
  b->total_pix = pix;
  b->total_samples = sample;
  b->tn = tn;
  int rc = wf_alloc(&b->wf, tn.capacity, pix, b->nee_mult);
  if(rc == DORT_OK && (dev_alloc(&b->d_jobs, n * sizeof(WfJob)) != cudaSuccess ||
                       dev_alloc(&b->d_images, size_t(pix) * 3 * sizeof(float)) != cudaSuccess)) {
    cudaGetLastError();
    rc = fail(DORT_ERR_OOM, "cudaMalloc for the batch failed");
  }
  if(rc == DORT_OK &&
     cudaMemcpy(b->d_jobs, jobs.data(), n * sizeof(WfJob), cudaMemcpyHostToDevice) != cudaSuccess) {
    rc = fail(DORT_ERR_CUDA, "copy of the batch job table failed");
  }
  if(rc == DORT_OK) {
    b->wf.dev.total_samples = b->total_samples;
    b->wf.dev.max_waves = wave_bound(b->total_samples, tn.capacity, b->max_depth, tn.max_waves);
    bool general = false;
    for(uint32_t j = 0; j < n; ++j) { general = general || scene_needs_general(scenes[j], params[j]); }
    rc = general ? wf_build_graph(&b->wf, JobTable<true>{b->d_jobs, n}, tn)
                 : wf_build_graph(&b->wf, JobTable<false>{b->d_jobs, n}, tn);
    b->wf.jobs_cached = b->d_jobs;
  }
  if(rc != DORT_OK) {
    wavefront_batch_destroy(b);
    return rc;
  }
  *out = b;
  return DORT_OK;
}

int wavefront_batch_render(WavefrontBatch* b, cudaStream_t st) {
  Wavefront* wf = &b->wf;
  wf_init<<<(std::max(wf->capacity, b->total_pix) + 255) / 256, 256, 0, st>>>(wf->dev,
                                                                              b->total_pix);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaGraphLaunch(wf->exec, st));
  wf_resolve_batch<<<(b->total_pix + 255) / 256, 256, 0, st>>>(wf->dev, b->d_jobs,
                                                               b->job_count, b->total_pix,
                                                               b->d_images);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

int wavefront_batch_image(WavefrontBatch* b, uint32_t job, const float** d_rgb, uint32_t* npix) {
  if(job >= b->job_count) { return fail(DORT_ERR_INVALID, "job index out of range"); }
  *d_rgb = b->d_images + 3 * size_t(b->film_offset[job]);
  *npix = b->npix[job];
  return DORT_OK;
}

int wavefront_batch_counters(WavefrontBatch* b, uint64_t* rays, uint32_t* waves,
                             uint32_t* error, cudaStream_t st) {
  return wavefront_counters_of(&b->wf, rays, waves, error, st);
}

}  // namespace dort_gpu
