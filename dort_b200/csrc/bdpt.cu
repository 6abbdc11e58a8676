// The "bdpt" renderer (BdptRenderer, bdpt_renderer.cpp:9-468) on the device,
// connection-parallel.  The pixel samples of a frame (W x H x iterations, in
// the order pixel + npix * sample) are taken in chunks; per chunk:
//
//   bdpt_light_walks,    one thread per sample: the light walk, then the
//   bdpt_camera_walks    camera walk, into device memory (structure of
//                        arrays, so a warp's stores are whole lines); the
//                        camera kernel appends the sample's (s, t)
//                        connections to one list per case (bdpt_pair_case)
//                        with one atomic per warp and case;
//   bdpt_connect_kernel  one launch per case, one thread per listed
//                        connection: its rays and its MIS weight
//                        (bdpt_connect, the host check's code); t = 1
//                        connections splat onto the film, the others store
//                        their weighted value in the sample's slot for (s, t);
//   bdpt_gather          one thread per sample: the slots summed in the host
//                        loop's (s, t) order, the sample kept if finite and
//                        non-negative (renderer.cpp:36-41) and added to its
//                        pixel with one float4 atomic (sum, count).
//
// A resolve pass adds the splats scaled by 1 / iterations (the film's
// splat_scale at the end of render, :21-31).  The random numbers of a
// connection are keyed by (seed, pixel, sample, s, t), so the image is the
// host check's up to float rounding and the order of the atomic sums.
//
// Against one thread per sample running both walks and every connection:
// a warp of a connection kernel runs one case's code on 32 connections
// instead of 32 samples' mixed (s, t) loops, each kernel's code fits the
// instruction cache, and the walks stay in device memory rather than
// per-thread local arrays read back by every MIS weight.
#include <algorithm>

#include "bdpt.cuh"
#include "common.h"

namespace dort_gpu {

constexpr int kBdptBlock = 128;
#ifndef DORT_BDPT_CHUNK_LOG2
#define DORT_BDPT_CHUNK_LOG2 20
#endif
// samples per chunk (< 2^24: the list entries' sample field); chunks of
// 2^21 or 2^22 samples measured the same on the Cornell workload
constexpr uint32_t kBdptChunk = 1u << DORT_BDPT_CHUNK_LOG2;
// Resident blocks per SM the register allocation must allow (Cornell
// workload, A/B against the compiler's 104-128 registers): connection
// kernels at 6 blocks +13 %, at 8 (64 registers, some spill) another +4 %;
// walk kernels at 5 (96 registers) +8 %, at 6 less.
#ifndef DORT_BDPT_CONNECT_MIN_BLOCKS
#define DORT_BDPT_CONNECT_MIN_BLOCKS 8
#endif
#ifndef DORT_BDPT_WALK_MIN_BLOCKS
#define DORT_BDPT_WALK_MIN_BLOCKS 5
#endif

// Connection slots of one sample: (s, t) with t >= 1 and s + t <= D =
// max_depth + 2, numbered in the host loop's order (s outer, t inner); at
// most D (D + 1) / 2 = 120 (max_depth <= 13).
DG_HD uint32_t bd_slot(uint32_t D, uint32_t s, uint32_t t) {
  return s * D - s * (s - 1) / 2 + t - 1;
}

// Per-sample capacity of each case's list for D = max_depth + 2: s = 0 with
// t = 2..D; s = 1 with t = 2..D-1; t = 1 with s = 1..D-1; s, t >= 2.
static uint32_t bd_case_cap(uint32_t D, uint32_t c) {
  switch(c) {
    case kBdCaseS0: return D - 1;
    case kBdCaseS1: return D >= 2 ? D - 2 : 0;
    case kBdCaseT1: return D - 1;
    default: return D >= 4 ? (D - 3) * (D - 2) / 2 : 0;
  }
}

struct BdptChunk {
  float4* lw;                 // light walks: SoaWalk, 5 D words per sample
  float4* cw;                 // camera walks
  uint4* rec0;                // pixel, sample, light index, ns | nt << 8
  float4* rec1;               // light pick probability, film x, film y, - (between
                              // the walk kernels: pick, light index, ns, -)
  uint4* mask;                // slots holding a t >= 2 connection's value
  float* contrib;             // slot values: ((slot * 3 + channel) * cap + i)
  uint32_t* list[kBdCases];   // connections: i << 8 | s << 4 | t
  uint32_t list_cap[kBdCases];  // entries each list holds (bd_case_cap x cap)
  uint32_t* count;            // list lengths
  uint32_t cap;               // samples per chunk
  uint32_t D;                 // max_depth + 2
};

__device__ __forceinline__ uint32_t bd_case_count(uint32_t packed, uint32_t c) {
  return (packed >> (8 * c)) & 0xffu;
}

// The light walks of a chunk: the light pick and the walk of each sample;
// rec1 carries the pick, the light's index and the vertex count to the
// camera walks.
template<bool G>
__global__ void __launch_bounds__(kBdptBlock, DORT_BDPT_WALK_MIN_BLOCKS)
bdpt_light_walks(PtScene sc, PtParams pp, uint64_t first, uint32_t count, BdptChunk ch,
                 unsigned long long* __restrict__ counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = pp.width * pp.height;
  uint32_t rays = 0;
  if(i < count) {
    const uint64_t g = first + i;
    const uint32_t pixel = uint32_t(g % npix), sample = uint32_t(g / npix);
    uint32_t light_i = 0, ns = 0;
    float pick = 0.f;
    if(sc.light_count != 0) {
      BdptCtx c{sc, pp, pixel, sample};
      Rand4 r1 = rand4(pp.seed, pixel, sample, 1);
      light_i = distrib_sample(sc.light_cdf, sc.light_count + 1, r1.a);
      pick = distrib_pdf(sc.light_cdf, sc.light_count + 1, light_i);
      const SoaWalk lw{ch.lw, ch.cap, i};
      ns = pick > 0.f ? bdpt_light_walk<G>(c, light_i, pick, lw, rays) : 0u;
      if(ns == 0) { lw.put(0, bvert_empty()); }
    }
    ch.rec1[i] = make_float4(pick, __uint_as_float(light_i), __uint_as_float(ns), 0.f);
  }
  unsigned long long r = rays;
  for(int o = 16; o > 0; o >>= 1) { r += __shfl_down_sync(0xffffffffu, r, o); }
  if((threadIdx.x & 31u) == 0 && r) { atomicAdd(&counters[0], r); }
}

// The camera walks of a chunk, then each sample's connections: counted per
// case, their slots marked for the gather, appended to the case lists.
template<bool G>
__global__ void __launch_bounds__(kBdptBlock, DORT_BDPT_WALK_MIN_BLOCKS)
bdpt_camera_walks(PtScene sc, PtParams pp, uint64_t first, uint32_t count, BdptChunk ch,
                  unsigned long long* __restrict__ counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < count;
  const uint32_t npix = pp.width * pp.height;
  const bool use_t1 = pp.use_t1 != 0;
  uint32_t rays = 0, ns = 0, nt = 0, emit = 0;
  if(valid) {
    const uint64_t g = first + i;
    const uint32_t pixel = uint32_t(g % npix), sample = uint32_t(g / npix);
    Rand4 r0 = rand4(pp.seed, pixel, sample, 0);
    const float fx = float(pixel % pp.width) + r0.a, fy = float(pixel / pp.width) + r0.b;
    const float4 lr = ch.rec1[i];
    const uint32_t light_i = __float_as_uint(lr.y);
    ns = __float_as_uint(lr.z);
    if(sc.light_count != 0) {
      BdptCtx c{sc, pp, pixel, sample};
      const SoaWalk cw{ch.cw, ch.cap, i};
      nt = bdpt_camera_walk<G>(c, fx, fy, cw, rays, emit);
    }
    ch.rec0[i] = make_uint4(pixel, sample, light_i, ns | (nt << 8));
    ch.rec1[i] = make_float4(lr.x, fx, fy, 0.f);
  }
  // the sample's connections: counts per case (8 bits each: at most 120)
  // and the slots the gather sums
  uint32_t packed = 0, m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  if(valid && nt > 0) {
    for(uint32_t s = 0; s <= ns; ++s) {
      for(uint32_t t = 1; t <= nt; ++t) {
        const uint32_t c = bdpt_pair_case(pp, use_t1, emit, s, t);
        if(c == kBdCases) { continue; }
        packed += 1u << (8 * c);
        if(t >= 2) {
          const uint32_t slot = bd_slot(ch.D, s, t), w = slot >> 5, b = 1u << (slot & 31u);
          m0 |= w == 0 ? b : 0u;
          m1 |= w == 1 ? b : 0u;
          m2 |= w == 2 ? b : 0u;
          m3 |= w == 3 ? b : 0u;
        }
      }
    }
  }
  if(valid) { ch.mask[i] = make_uint4(m0, m1, m2, m3); }
  // one atomic per warp and case: each lane's first entry in each list
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t off[kBdCases];
#pragma unroll
  for(uint32_t c = 0; c < kBdCases; ++c) {
    const uint32_t mine = bd_case_count(packed, c);
    uint32_t incl = mine;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if(lane >= uint32_t(o)) { incl += v; }
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if(lane == 31 && total) { base = atomicAdd(&ch.count[c], total); }
    base = __shfl_sync(0xffffffffu, base, 31);
    off[c] = base + incl - mine;
  }
  if(valid && packed) {
    for(uint32_t s = 0; s <= ns; ++s) {
      for(uint32_t t = 1; t <= nt; ++t) {
        const uint32_t c = bdpt_pair_case(pp, use_t1, emit, s, t);
        if(c == kBdCases) { continue; }
        const uint32_t code = (i << 8) | (s << 4) | t;
        // list and position by case, without indexing an array by c
        uint32_t* dst;
        uint32_t at;
        uint32_t lim;
        if(c == kBdCaseS0) {
          dst = ch.list[0]; at = off[0]++; lim = ch.list_cap[0];
        } else if(c == kBdCaseS1) {
          dst = ch.list[1]; at = off[1]++; lim = ch.list_cap[1];
        } else if(c == kBdCaseT1) {
          dst = ch.list[2]; at = off[2]++; lim = ch.list_cap[2];
        } else {
          dst = ch.list[3]; at = off[3]++; lim = ch.list_cap[3];
        }
        // the capacities bound every sample's count per case, so this never
        // skips; it keeps a wrong count from writing past the list
        if(at < lim) { dst[at] = code; }
      }
    }
  }
  unsigned long long r = rays;
  for(int o = 16; o > 0; o >>= 1) { r += __shfl_down_sync(0xffffffffu, r, o); }
  if(lane == 0 && r) { atomicAdd(&counters[0], r); }
}

template<bool G, uint32_t CASE>
__global__ void __launch_bounds__(kBdptBlock, DORT_BDPT_CONNECT_MIN_BLOCKS)
bdpt_connect_kernel(PtScene sc, PtParams pp, BdptChunk ch, float* __restrict__ splat,
                    unsigned long long* __restrict__ counters) {
  const uint32_t n = min(*(volatile uint32_t*)&ch.count[CASE], ch.list_cap[CASE]);
  const uint32_t* __restrict__ list = ch.list[CASE];
  uint32_t rays = 0;
  for(uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const uint32_t code = __ldg(&list[e]);
    const uint32_t i = code >> 8, s = (code >> 4) & 15u, t = code & 15u;
    const uint4 r0 = __ldg(&ch.rec0[i]);
    const float4 r1 = __ldg(&ch.rec1[i]);
    BdptCtx c{sc, pp, r0.x, r0.y};
    const SoaWalk lw{ch.lw, ch.cap, i}, cw{ch.cw, ch.cap, i};
    const BdptSampleData sd{r0.w & 0xffu, r0.w >> 8, r0.z, r1.x, r1.y, r1.z};
    V3 wc;
    float sfx, sfy;
    const bool ok = bdpt_connect<G, CASE>(c, lw, cw, sd, s, t, wc, sfx, sfy, rays);
    if constexpr(CASE == kBdCaseT1) {
      if(ok) { lt_splat(splat, pp, sfx, sfy, wc); }
    } else {
      if(!ok) { wc = v3(0.f, 0.f, 0.f); }
      float* q = ch.contrib + size_t(bd_slot(ch.D, s, t)) * 3 * ch.cap + i;
      q[0] = wc.x;
      q[ch.cap] = wc.y;
      q[2 * size_t(ch.cap)] = wc.z;
    }
  }
  unsigned long long r = rays;
  for(int o = 16; o > 0; o >>= 1) { r += __shfl_down_sync(0xffffffffu, r, o); }
  if((threadIdx.x & 31u) == 0 && r) { atomicAdd(&counters[0], r); }
}

__global__ void __launch_bounds__(kBdptBlock)
bdpt_gather(BdptChunk ch, uint32_t count, float4* __restrict__ acc,
            unsigned long long* __restrict__ counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long kept = 0;
  if(i < count) {
    const uint4 m = ch.mask[i];
    const uint32_t words[4] = {m.x, m.y, m.z, m.w};
    float lx = 0.f, ly = 0.f, lz = 0.f;
#pragma unroll
    for(uint32_t w = 0; w < 4; ++w) {
      uint32_t bits = words[w];
      while(bits) {
        const uint32_t slot = 32 * w + __ffs(bits) - 1;
        bits &= bits - 1;
        const float* q = ch.contrib + size_t(slot) * 3 * ch.cap + i;
        lx = lx + q[0];
        ly = ly + q[ch.cap];
        lz = lz + q[2 * size_t(ch.cap)];
      }
    }
    if(isfinite(lx) && isfinite(ly) && isfinite(lz) && lx >= 0.f && ly >= 0.f && lz >= 0.f) {
      atomicAdd(&acc[ch.rec0[i].x], make_float4(lx, ly, lz, 1.f));
      kept = 1;
    }
  }
  for(int o = 16; o > 0; o >>= 1) { kept += __shfl_down_sync(0xffffffffu, kept, o); }
  if((threadIdx.x & 31u) == 0 && kept) { atomicAdd(&counters[1], kept); }
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

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Blocks of a grid-stride connection launch: every resident block of the
// kernel on every SM.
template<uint32_t CASE>
static int connect_blocks(int sms) {
  // computed once (a thread-safe static initialiser)
  static const int per_sm = [] {
    int b = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, bdpt_connect_kernel<true, CASE>,
                                                     kBdptBlock, 0) != cudaSuccess || b < 1) {
      cudaGetLastError();
      b = 4;
    }
    return b;
  }();
  return per_sm * sms;
}

int launch_bdpt(dort_scene* s, const PtParams& pp, float* d_out, cudaStream_t st,
                unsigned long long* d_counters) {
  int dev = 0, sms = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t npix = size_t(pp.width) * pp.height;
  const uint64_t total = uint64_t(npix) * pp.spp;
  const uint32_t D = pp.max_depth + 2;   // <= 15: max_depth <= 13 (make_params)
  const uint32_t cap = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(total, kBdptChunk)));
  const uint32_t slots = D * (D + 1) / 2;
  // layout of the scratch: film sums, splats, then the chunk's buffers
  size_t off = 0;
  const size_t acc_off = off; off = align256(off + npix * sizeof(float4));
  const size_t splat_off = off; off = align256(off + npix * 3 * sizeof(float));
  const size_t walk_bytes = size_t(5) * D * cap * sizeof(float4);
  const size_t lw_off = off; off = align256(off + walk_bytes);
  const size_t cw_off = off; off = align256(off + walk_bytes);
  const size_t rec0_off = off; off = align256(off + size_t(cap) * sizeof(uint4));
  const size_t rec1_off = off; off = align256(off + size_t(cap) * sizeof(float4));
  const size_t mask_off = off; off = align256(off + size_t(cap) * sizeof(uint4));
  const size_t contrib_off = off; off = align256(off + size_t(slots) * 3 * cap * sizeof(float));
  size_t list_off[kBdCases];
  for(uint32_t c = 0; c < kBdCases; ++c) {
    list_off[c] = off;
    off = align256(off + size_t(std::max(1u, bd_case_cap(D, c))) * cap * sizeof(uint32_t));
  }
  const size_t count_off = off; off = align256(off + kBdCases * sizeof(uint32_t));
  void* scratch = nullptr;
  int rc = render_scratch(s, off, &scratch);
  if(rc != DORT_OK) { return rc; }
  char* base = static_cast<char*>(scratch);
  float4* acc = reinterpret_cast<float4*>(base + acc_off);
  float* splat = reinterpret_cast<float*>(base + splat_off);
  BdptChunk ch;
  ch.lw = reinterpret_cast<float4*>(base + lw_off);
  ch.cw = reinterpret_cast<float4*>(base + cw_off);
  ch.rec0 = reinterpret_cast<uint4*>(base + rec0_off);
  ch.rec1 = reinterpret_cast<float4*>(base + rec1_off);
  ch.mask = reinterpret_cast<uint4*>(base + mask_off);
  ch.contrib = reinterpret_cast<float*>(base + contrib_off);
  for(uint32_t c = 0; c < kBdCases; ++c) {
    ch.list[c] = reinterpret_cast<uint32_t*>(base + list_off[c]);
    ch.list_cap[c] = std::max(1u, bd_case_cap(D, c)) * cap;
  }
  ch.count = reinterpret_cast<uint32_t*>(base + count_off);
  ch.cap = cap;
  ch.D = D;
  DG_CUDA(cudaMemsetAsync(base, 0, lw_off, st));   // film sums and splats
  // one instantiation: the bidirectional tracer is not specialised (the
  // triangle-only instantiation of the same kernels, chosen per scene like
  // the path tracer's, rendered the Cornell workload's identical image at
  // 139.6 against 212.2 M samples/s)
  for(uint64_t first = 0; first < total; first += cap) {
    const uint32_t count = uint32_t(std::min<uint64_t>(cap, total - first));
    DG_CUDA(cudaMemsetAsync(ch.count, 0, kBdCases * sizeof(uint32_t), st));
    const uint32_t blocks = (count + kBdptBlock - 1) / kBdptBlock;
    bdpt_light_walks<true><<<blocks, kBdptBlock, 0, st>>>(s->pt, pp, first, count, ch,
                                                          d_counters);
    bdpt_camera_walks<true><<<blocks, kBdptBlock, 0, st>>>(s->pt, pp, first, count, ch,
                                                           d_counters);
    DG_CUDA(cudaGetLastError());
    bdpt_connect_kernel<true, kBdCaseS0><<<connect_blocks<kBdCaseS0>(sms), kBdptBlock, 0, st>>>(
        s->pt, pp, ch, splat, d_counters);
    bdpt_connect_kernel<true, kBdCaseS1><<<connect_blocks<kBdCaseS1>(sms), kBdptBlock, 0, st>>>(
        s->pt, pp, ch, splat, d_counters);
    bdpt_connect_kernel<true, kBdCaseT1><<<connect_blocks<kBdCaseT1>(sms), kBdptBlock, 0, st>>>(
        s->pt, pp, ch, splat, d_counters);
    bdpt_connect_kernel<true, kBdCaseST><<<connect_blocks<kBdCaseST>(sms), kBdptBlock, 0, st>>>(
        s->pt, pp, ch, splat, d_counters);
    DG_CUDA(cudaGetLastError());
    bdpt_gather<<<blocks, kBdptBlock, 0, st>>>(ch, count, acc, d_counters);
    DG_CUDA(cudaGetLastError());
  }
  bdpt_resolve<<<uint32_t((npix + 255) / 256), 256, 0, st>>>(acc, splat, uint32_t(npix),
                                                             1.f / float(pp.spp), d_out);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

}  // namespace dort_gpu
