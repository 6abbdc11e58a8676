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
#include <algorithm>
#include <cstring>
#include <string>

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
  C_NEXT_LO = 16,   // 64-bit next-sample counter at [16..17]
  C_RAYS_LO = 18,   // 64-bit ray counter at [18..19]
  C_COUNT = 32
};

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

// Maps a global sample id to (pixel, x, y, sample): sample-major order, 8x4
// pixel tiles, so consecutive ids are coherent primary rays.
__device__ __forceinline__ void sample_to_pixel(const PtParams& pp, uint64_t sid,
                                                uint32_t& pixel, uint32_t& x, uint32_t& y,
                                                uint32_t& s) {
  uint32_t tiles_x = (pp.width + 7) / 8;
  uint32_t tiles = tiles_x * ((pp.height + 3) / 4);
  uint64_t per_sample = uint64_t(tiles) * 32;
  s = uint32_t(sid / per_sample);
  uint32_t local = uint32_t(sid % per_sample);
  uint32_t tile = local / 32, lane = local % 32;
  x = (tile % tiles_x) * 8 + lane % 8;
  y = (tile / tiles_x) * 4 + lane / 8;
  pixel = y * pp.width + x;
}

struct WfDev {
  float4* ray_o;   // o.xyz, t_min
  float4* ray_d;   // d.xyz, -
  float4* thr;     // throughput
  float4* sum;     // radiance sum
  uint4* meta;     // pixel, sample, bounces | last_delta << 31, state
  float4* hit;     // t, b1, b2, prim
  uint32_t* active[2];
  uint32_t* finished[2];
  uint32_t* sh_slot;
  float4* sh_o;    // o.xyz, t_min
  float4* sh_d;    // d.xyz, t_max
  float4* sh_c;    // contribution
  uint32_t* nb_slot;
  float4* nb_o;    // o.xyz, t_min
  float4* nb_d;    // d.xyz, pdf
  float4* nb_f;    // factor.xyz, light index (bits) | use_mis << 31
  float4* film;    // sum rgb, kept count
  uint32_t* ctr;
  uint32_t capacity;
  uint64_t total_samples;
  uint32_t max_waves;
};

__device__ __forceinline__ uint32_t wave_of(const WfDev& w) {
  return *(volatile uint32_t*)(w.ctr + C_WAVES);
}

__global__ void wf_init(WfDev w, uint32_t npix) {
  uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < w.capacity; i += stride) {
    w.meta[i] = make_uint4(0u, 0u, 0u, SLOT_FREE);
    w.finished[0][i] = uint32_t(i);    // every slot starts on the free list
  }
  for(uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < npix; i += stride) {
    w.film[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if(blockIdx.x == 0 && threadIdx.x < C_COUNT) {
    w.ctr[threadIdx.x] = threadIdx.x == C_FIN0 ? w.capacity : 0u;
  }
}

// Finished paths of the last wave go to the film; their slots (and, in the
// first wave, every slot) take the next samples and join this wave's active
// queue behind the paths that continue.
__global__ void wf_regen(PtScene sc, PtParams pp, WfDev w) {
  const uint32_t wave = wave_of(w);
  const uint32_t cur = wave & 1u;
  const uint32_t n = *(volatile uint32_t*)(w.ctr + C_FIN0 + cur);
  const uint32_t* fin = w.finished[cur];
  uint32_t* act = w.active[cur];
  uint64_t* next = reinterpret_cast<uint64_t*>(w.ctr + C_NEXT_LO);
  uint32_t stride = gridDim.x * blockDim.x;
  uint32_t n_pad = (n + 31u) & ~31u;
  for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
    bool valid = i < n;
    uint32_t slot = valid ? fin[i] : 0u;
    uint4 m = valid ? w.meta[slot] : make_uint4(0u, 0u, 0u, SLOT_ACTIVE);
    if(valid && m.w == SLOT_FINISHED) {
      float4 s = w.sum[slot];
      // renderer.cpp:36-41: only finite, non-negative samples reach the film
      bool keep = isfinite(s.x) && isfinite(s.y) && isfinite(s.z) && s.x >= 0.f &&
                  s.y >= 0.f && s.z >= 0.f;
      if(keep) { atomicAdd(w.film + m.x, make_float4(s.x, s.y, s.z, 1.f)); }
      atomicSub(w.ctr + C_LIVE, 1u);
      m.w = SLOT_FREE;
    }
    bool want_new = valid && m.w == SLOT_FREE;
    uint32_t nmask = __ballot_sync(0xffffffffu, want_new);
    uint64_t sid = ~0ull;
    if(want_new) {
      uint32_t lane = threadIdx.x & 31u, leader = __ffs(nmask) - 1u;
      unsigned long long base = 0;
      if(lane == leader) {
        base = atomicAdd(reinterpret_cast<unsigned long long*>(next),
                         (unsigned long long)__popc(nmask));
      }
      base = __shfl_sync(nmask, base, leader);
      sid = base + __popc(nmask & ((1u << lane) - 1u));
    }
    bool fresh = false;
    if(want_new && sid < w.total_samples) {
      uint32_t pixel, x, y, s;
      sample_to_pixel(pp, sid, pixel, x, y, s);
      if(x < pp.width && y < pp.height) {
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
        camera_ray(pp, fx, fy, o, d);
        w.ray_o[slot] = make_float4(o.x, o.y, o.z, 0.f);
        w.ray_d[slot] = make_float4(d.x, d.y, d.z, 0.f);
        w.thr[slot] = make_float4(1.f, 1.f, 1.f, 0.f);
        w.sum[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
        m = make_uint4(pixel, s, 0u, SLOT_ACTIVE);
        fresh = true;
      }
    }
    if(want_new) { w.meta[slot] = m; }
    if(fresh) { atomicAdd(w.ctr + C_LIVE, 1u); }
    // a slot whose sample fell outside the image goes back on the next free
    // list so that it keeps taking samples
    bool retry = want_new && !fresh && sid < w.total_samples;
    uint32_t at = warp_append(w.ctr + C_ACT0 + cur, fresh);
    if(fresh) { act[at] = slot; }
    uint32_t rt = warp_append(w.ctr + C_FIN0 + (cur ^ 1u), retry);
    if(retry) { w.finished[cur ^ 1u][rt] = slot; }
  }
}

__global__ void wf_extend(PtScene sc, WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  const uint32_t n = *(volatile uint32_t*)(w.ctr + C_ACT0 + cur);
  const uint32_t* act = w.active[cur];
  for(;;) {
    uint32_t base = warp_fetch(w.ctr + C_F_EXT);
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    if(i < n) {
      uint32_t slot = act[i];
      float4 o = w.ray_o[slot], d = w.ray_d[slot];
      Hit h = trace_ray<false>(sc.trace, o.x, o.y, o.z, o.w, d.x, d.y, d.z, INFINITY);
      w.hit[slot] = make_float4(h.t, h.b1, h.b2, u2f(h.prim));
    }
  }
}

__global__ void wf_shade(PtScene sc, PtParams pp, WfDev w) {
  const uint32_t cur = wave_of(w) & 1u;
  const uint32_t n = *(volatile uint32_t*)(w.ctr + C_ACT0 + cur);
  const uint32_t* act = w.active[cur];
  uint32_t* act_next = w.active[cur ^ 1u];
  uint32_t* fin_next = w.finished[cur ^ 1u];
  const uint32_t req_nd = F_ALL & ~F_DELTA;
  for(;;) {
    uint32_t base = warp_fetch(w.ctr + C_F_SHADE);
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    bool valid = i < n;
    bool push_sh = false, push_nb = false, cont = false, done = false;
    float4 sh_o, sh_d, sh_c, nb_o, nb_d, nb_f;
    uint32_t slot = 0;
    if(valid) {
      slot = act[i];
      float4 ro = w.ray_o[slot], rd = w.ray_d[slot];
      float4 t4 = w.thr[slot], s4 = w.sum[slot];
      uint4 m = w.meta[slot];
      float4 h4 = w.hit[slot];
      Hit h;
      h.t = h4.x; h.b1 = h4.y; h.b2 = h4.z; h.prim = f2u(h4.w);
      V3 o = v3(ro.x, ro.y, ro.z), d = v3(rd.x, rd.y, rd.z);
      V3 thr = v3(t4.x, t4.y, t4.z), sum = v3(s4.x, s4.y, s4.z);
      uint32_t bounces = m.z & 0x7fffffffu;
      bool last_delta = (m.z >> 31) != 0;
      bool hit = h.prim != kMiss;
      SurfaceHit g;
      if(hit) { g = surface_at(sc, h); }
      if((bounces == 0 || last_delta) && bounces >= pp.min_depth && bounces <= pp.max_depth) {
        if(hit) {
          if(g.light) {
            const DevLight& l = sc.lights[g.light - 1];
            sum = sum + thr * area_eval_radiance(sc, l, g.p, g.n, o);
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
        uint32_t blk = bounce_block(bounces);
        Rand4 r0 = rand4(pp.seed, m.x, m.y, blk);
        Rand4 r1 = rand4(pp.seed, m.x, m.y, blk + 1);
        Rand4 r2 = rand4(pp.seed, m.x, m.y, blk + 2);
        if(bounces >= pp.min_depth && bxdf_matches(mt.bxdf_flags, req_nd) && sc.light_count > 0) {
          uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, r0.a);
          float lpdf = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
          if(lpdf != 0.f) {
            const DevLight& l = sc.lights[li];
            bool use_bsdf = pp.strategy != 2, use_light = pp.strategy != 1;
            if(use_bsdf) {
              BsdfSample bs = bsdf_sample(mt, g.frame, wo, req_nd, r0.b, r0.c, r0.d);
              if(!(bs.pdf == 0.f || is_black(bs.f))) {
                // contribution = f * L * (w |n.wi| / pdf) * thr / light_pick_pdf,
                // L and w known once the ray is traced
                V3 fac = thr * (bs.f * (fabsf(dot(g.n, bs.w)) / bs.pdf)) * (1.f / lpdf);
                push_nb = true;
                nb_o = make_float4(g.p.x, g.p.y, g.p.z, g.eps);
                nb_d = make_float4(bs.w.x, bs.w.y, bs.w.z, bs.pdf);
                nb_f = make_float4(fac.x, fac.y, fac.z, u2f(li | (use_light ? 0x80000000u : 0u)));
              }
            }
            if(use_light) {
              LightSample ls = light_sample(sc, l, g.p, g.eps, r1.a, r1.b);
              if(!(ls.pdf == 0.f || is_black(ls.L))) {
                V3 f = bsdf_eval(mt, g.frame, ls.wi, wo, req_nd);
                if(!is_black(f)) {
                  float wgt = 1.f;
                  if(use_bsdf) {
                    float bp = bsdf_pdf(mt, g.frame, ls.wi, wo, req_nd);
                    wgt = ls.pdf / (ls.pdf + bp);
                  }
                  V3 c = (f * ls.L * (wgt * fabsf(dot(g.n, ls.wi)) / ls.pdf)) * (1.f / lpdf) * thr;
                  push_sh = true;
                  sh_o = make_float4(ls.o.x, ls.o.y, ls.o.z, ls.tmin);
                  sh_d = make_float4(ls.d.x, ls.d.y, ls.d.z, ls.tmax);
                  sh_c = make_float4(c.x, c.y, c.z, 0.f);
                }
              }
            }
          }
        }
        uint32_t req = (pp.only_direct || bounces == pp.max_depth) ? (F_MODES | F_DELTA) : F_ALL;
        BsdfSample bs = bsdf_sample(mt, g.frame, wo, req, r1.c, r1.d, r2.a);
        if(is_black(bs.f) || bs.pdf == 0.f) {
          finished = true;
        } else {
          V3 contrib = bs.f * (fabsf(dot(bs.w, g.n)) / bs.pdf);
          last_delta = (bs.flags & F_DELTA) != 0;
          thr = thr * contrib;
          if(bounces == pp.max_depth && !last_delta) {
            finished = true;
          } else if(bounces >= 2 && bounces > pp.min_depth) {
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
          }
        }
      }
      w.sum[slot] = make_float4(sum.x, sum.y, sum.z, 0.f);
      m.z = bounces | (last_delta ? 0x80000000u : 0u);
      m.w = finished ? SLOT_FINISHED : SLOT_ACTIVE;
      w.meta[slot] = m;
      cont = !finished;
      done = finished;
    }
    uint32_t ci = warp_append(w.ctr + C_ACT0 + (cur ^ 1u), cont);
    if(cont) { act_next[ci] = slot; }
    uint32_t fi = warp_append(w.ctr + C_FIN0 + (cur ^ 1u), done);
    if(done) { fin_next[fi] = slot; }
    uint32_t si = warp_append(w.ctr + C_SHADOW, push_sh);
    if(push_sh) {
      w.sh_slot[si] = slot;
      w.sh_o[si] = sh_o;
      w.sh_d[si] = sh_d;
      w.sh_c[si] = sh_c;
    }
    uint32_t ni = warp_append(w.ctr + C_NEEB, push_nb);
    if(push_nb) {
      w.nb_slot[ni] = slot;
      w.nb_o[ni] = nb_o;
      w.nb_d[ni] = nb_d;
      w.nb_f[ni] = nb_f;
    }
  }
}

__global__ void wf_shadow(PtScene sc, WfDev w) {
  const uint32_t n = *(volatile uint32_t*)(w.ctr + C_SHADOW);
  for(;;) {
    uint32_t base = warp_fetch(w.ctr + C_F_SH);
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    if(i < n) {
      float4 o = w.sh_o[i], d = w.sh_d[i];
      Hit h = trace_ray<true>(sc.trace, o.x, o.y, o.z, o.w, d.x, d.y, d.z, d.w);
      if(h.prim == kMiss) {
        uint32_t slot = w.sh_slot[i];
        float4 c = w.sh_c[i];
        float4 s = w.sum[slot];
        w.sum[slot] = make_float4(s.x + c.x, s.y + c.y, s.z + c.z, 0.f);
      }
    }
  }
}

__device__ __forceinline__ void neeb_one_impl(const PtScene& sc, WfDev& w, uint32_t i);
#define neeb_one neeb_one_impl

__global__ void wf_neeb(PtScene sc, WfDev w) {
  const uint32_t n = *(volatile uint32_t*)(w.ctr + C_NEEB);
  for(;;) {
    uint32_t base = warp_fetch(w.ctr + C_F_NB);
    if(base >= n) { break; }
    uint32_t i = base + (threadIdx.x & 31u);
    if(i < n) { neeb_one(sc, w, i); }
  }
}

__device__ __forceinline__ void neeb_one_impl(const PtScene& sc, WfDev& w, uint32_t i) {
    float4 o = w.nb_o[i], d = w.nb_d[i], f = w.nb_f[i];
    uint32_t lw = f2u(f.w);
    const DevLight& l = sc.lights[lw & 0x7fffffffu];
    bool use_mis = (lw >> 31) != 0;
    V3 L = v3(0.f, 0.f, 0.f);
    V3 p = v3(o.x, o.y, o.z), wi = v3(d.x, d.y, d.z);
    if(l.kind == LIGHT_TRI) {
      Hit h = trace_ray<false>(sc.trace, o.x, o.y, o.z, o.w, d.x, d.y, d.z, INFINITY);
      if(h.prim != kMiss && h.prim == l.tri) {
        const float4* sh = sc.shade + 3 * size_t(h.prim);
        float4 a = sh[0], b = sh[1], c = sh[2];
        V3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
        float b0 = 1.f - h.b1 - h.b2;
        V3 lp = b0 * p0 + h.b1 * p1 + h.b2 * p2;
        V3 ln = normalize(cross(p2 - p0, p1 - p0));
        L = area_eval_radiance(sc, l, lp, ln, p);
      }
    } else {
      // background light: only escaping rays count, an any-hit query decides
      Hit h = trace_ray<true>(sc.trace, o.x, o.y, o.z, o.w, d.x, d.y, d.z, INFINITY);
      if(h.prim == kMiss) { L = background_radiance(sc, l, wi); }
    }
    if(!is_black(L)) {
      float wgt = 1.f;
      if(use_mis) {
        float lp = light_pivot_pdf(sc, l, wi, p);
        wgt = d.w / (d.w + lp);
      }
      V3 c = v3(f.x, f.y, f.z) * L * wgt;
      uint32_t slot = w.nb_slot[i];
      float4 s = w.sum[slot];
      w.sum[slot] = make_float4(s.x + c.x, s.y + c.y, s.z + c.z, 0.f);
    }
}

// Single thread: account the wave, retire its queues, decide whether to loop.
__device__ __forceinline__ bool wf_end_wave(WfDev& w) {
  uint32_t wave = w.ctr[C_WAVES];
  uint32_t cur = wave & 1u;
  uint32_t a = w.ctr[C_ACT0 + cur], s = w.ctr[C_SHADOW], b = w.ctr[C_NEEB];
  unsigned long long* rays = reinterpret_cast<unsigned long long*>(w.ctr + C_RAYS_LO);
  *rays += (unsigned long long)a + s + b;
  w.ctr[C_ACT0 + cur] = 0u;     // consumed; the next wave fills the other buffer
  w.ctr[C_FIN0 + cur] = 0u;
  w.ctr[C_SHADOW] = 0u;
  w.ctr[C_NEEB] = 0u;
  w.ctr[C_F_EXT] = 0u;
  w.ctr[C_F_SHADE] = 0u;
  w.ctr[C_F_SH] = 0u;
  w.ctr[C_F_NB] = 0u;
  w.ctr[C_WAVES] = wave + 1u;
  uint64_t next = *reinterpret_cast<uint64_t*>(w.ctr + C_NEXT_LO);
  bool more = w.ctr[C_LIVE] > 0u || next < w.total_samples;
  if(more && wave + 1u >= w.max_waves) {
    // bounded: a frame never loops forever; the host reports the error
    w.ctr[C_ERROR] = 1u;
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

// ---- host side --------------------------------------------------------------------

struct Wavefront {
  WfDev dev{};
  cudaStream_t capture_stream = nullptr;   // graphs cannot be captured on stream 0
  void* mem = nullptr;
  size_t mem_bytes = 0;
  uint32_t capacity = 0;
  uint32_t npix_cap = 0;
  // graph cache (rebuilt when parameters change)
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  PtParams pp_cached{};
  WfTuning tune_cached{};
  bool valid = false;
};

static void wf_release(Wavefront* wf) {
  if(wf->capture_stream) { cudaStreamDestroy(wf->capture_stream); wf->capture_stream = nullptr; }
  if(wf->exec) { cudaGraphExecDestroy(wf->exec); wf->exec = nullptr; }
  if(wf->graph) { cudaGraphDestroy(wf->graph); wf->graph = nullptr; }
  if(wf->mem) { cudaFree(wf->mem); wf->mem = nullptr; }
  wf->valid = false;
}

void wavefront_destroy(Wavefront* wf) {
  if(!wf) { return; }
  wf_release(wf);
  delete wf;
}

static int wf_alloc(Wavefront* wf, uint32_t capacity, uint32_t npix) {
  if(wf->mem && wf->capacity == capacity && wf->npix_cap >= npix) { return DORT_OK; }
  wf_release(wf);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t Q = capacity;
  size_t f4 = al(Q * sizeof(float4)), u4 = al(Q * sizeof(uint4)), u1 = al(Q * sizeof(uint32_t));
  size_t bytes = 4 * f4 + u4 + f4 /*hit*/ + 4 * u1 /*active, finished*/ + u1 +
                 3 * f4 /*shadow*/ + u1 + 3 * f4 /*neeb*/ +
                 al(size_t(npix) * sizeof(float4)) + al(C_COUNT * 4);
  if(cudaMalloc(&wf->mem, bytes) != cudaSuccess) {
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
  d.meta = reinterpret_cast<uint4*>(take(u4));
  d.hit = reinterpret_cast<float4*>(take(f4));
  d.active[0] = reinterpret_cast<uint32_t*>(take(u1));
  d.active[1] = reinterpret_cast<uint32_t*>(take(u1));
  d.finished[0] = reinterpret_cast<uint32_t*>(take(u1));
  d.finished[1] = reinterpret_cast<uint32_t*>(take(u1));
  d.sh_slot = reinterpret_cast<uint32_t*>(take(u1));
  d.sh_o = reinterpret_cast<float4*>(take(f4));
  d.sh_d = reinterpret_cast<float4*>(take(f4));
  d.sh_c = reinterpret_cast<float4*>(take(f4));
  d.nb_slot = reinterpret_cast<uint32_t*>(take(u1));
  d.nb_o = reinterpret_cast<float4*>(take(f4));
  d.nb_d = reinterpret_cast<float4*>(take(f4));
  d.nb_f = reinterpret_cast<float4*>(take(f4));
  d.film = reinterpret_cast<float4*>(take(al(size_t(npix) * sizeof(float4))));
  d.ctr = reinterpret_cast<uint32_t*>(take(al(C_COUNT * 4)));
  d.capacity = capacity;
  wf->capacity = capacity;
  wf->npix_cap = npix;
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

static int wf_build_graph(Wavefront* wf, const PtScene& sc, const PtParams& pp,
                          const WfTuning& tn) {
  if(!wf->capture_stream) {
    DG_CUDA(cudaStreamCreateWithFlags(&wf->capture_stream, cudaStreamNonBlocking));
  }
  cudaStream_t st = wf->capture_stream;
  if(wf->exec) { cudaGraphExecDestroy(wf->exec); wf->exec = nullptr; }
  if(wf->graph) { cudaGraphDestroy(wf->graph); wf->graph = nullptr; }
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

  int b_trace = int(tn.trace_block), b_shade = int(tn.shade_block);
  int g_regen = grid_for(reinterpret_cast<const void*>(&wf_regen), 256);
  int g_ext = grid_for(reinterpret_cast<const void*>(&wf_extend), b_trace);
  int g_sha = grid_for(reinterpret_cast<const void*>(&wf_shade), b_shade);
  int g_shw = grid_for(reinterpret_cast<const void*>(&wf_shadow), b_trace);
  int g_nb = grid_for(reinterpret_cast<const void*>(&wf_neeb), b_trace);

  DG_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  wf_regen<<<g_regen, 256, 0, st>>>(sc, pp, wf->dev);
  wf_extend<<<g_ext, b_trace, 0, st>>>(sc, wf->dev);
  wf_shade<<<g_sha, b_shade, 0, st>>>(sc, pp, wf->dev);
  wf_shadow<<<g_shw, b_trace, 0, st>>>(sc, wf->dev);
  wf_neeb<<<g_nb, b_trace, 0, st>>>(sc, wf->dev);
  wf_control<<<1, 1, 0, st>>>(wf->dev, handle);
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(st, &captured);
  if(ce != cudaSuccess) {
    return fail(DORT_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(ce));
  }
  DG_CUDA(cudaGraphInstantiate(&wf->exec, wf->graph, 0));
  wf->pp_cached = pp;
  wf->tune_cached = tn;
  wf->valid = true;
  return DORT_OK;
}

static bool same_params(const PtParams& a, const PtParams& b) {
  return std::memcmp(&a, &b, sizeof(PtParams)) == 0;
}

int wavefront_render(dort_scene* s, const PtParams& pp, const WfTuning& tn, float* d_out,
                     cudaStream_t st) {
  if(!s->wavefront) { s->wavefront = new Wavefront(); }
  Wavefront* wf = s->wavefront;
  uint32_t npix = pp.width * pp.height;
  int rc = wf_alloc(wf, tn.capacity, npix);
  if(rc != DORT_OK) { return rc; }
  uint32_t tiles = ((pp.width + 7) / 8) * ((pp.height + 3) / 4);
  wf->dev.total_samples = uint64_t(tiles) * 32 * pp.spp;
  wf->dev.max_waves = uint32_t(std::min<uint64_t>(
      0x7fffffffull, (wf->dev.total_samples / std::max(1u, tn.capacity) + 2) *
                     (uint64_t(pp.max_depth) + 3) + 64));
  if(!wf->valid || !same_params(wf->pp_cached, pp) ||
     std::memcmp(&wf->tune_cached, &tn, sizeof(WfTuning)) != 0) {
    rc = wf_build_graph(wf, s->pt, pp, tn);
    if(rc != DORT_OK) { return rc; }
  }
  // the graph holds the kernel arguments, including total_samples and max_waves
  wf_init<<<(std::max(tn.capacity, npix) + 255) / 256, 256, 0, st>>>(wf->dev, npix);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaGraphLaunch(wf->exec, st));
  wf_resolve<<<(npix + 255) / 256, 256, 0, st>>>(wf->dev, npix, d_out);
  DG_CUDA(cudaGetLastError());
  return DORT_OK;
}

// The same frame as wavefront_render, run wave by wave from the host without
// the graph, with CUDA events around every stage; for measurement only.
__global__ void wf_control_host(WfDev w, uint32_t* more_flag) {
  *more_flag = wf_end_wave(w) ? 1u : 0u;
}

int wavefront_stage_times(dort_scene* s, const PtParams& pp, const WfTuning& tn,
                          float* d_out, cudaStream_t st, double ms[6]) {
  if(!s->wavefront) { s->wavefront = new Wavefront(); }
  Wavefront* wf = s->wavefront;
  uint32_t npix = pp.width * pp.height;
  int rc = wf_alloc(wf, tn.capacity, npix);
  if(rc != DORT_OK) { return rc; }
  uint32_t tiles = ((pp.width + 7) / 8) * ((pp.height + 3) / 4);
  wf->dev.total_samples = uint64_t(tiles) * 32 * pp.spp;
  wf->dev.max_waves = uint32_t(std::min<uint64_t>(
      0x7fffffffull, (wf->dev.total_samples / std::max(1u, tn.capacity) + 2) *
                     (uint64_t(pp.max_depth) + 3) + 64));
  const PtScene& sc = s->pt;
  int b_trace = int(tn.trace_block), b_shade = int(tn.shade_block);
  int g_regen = grid_for(reinterpret_cast<const void*>(&wf_regen), 256);
  int g_ext = grid_for(reinterpret_cast<const void*>(&wf_extend), b_trace);
  int g_sha = grid_for(reinterpret_cast<const void*>(&wf_shade), b_shade);
  int g_shw = grid_for(reinterpret_cast<const void*>(&wf_shadow), b_trace);
  int g_nb = grid_for(reinterpret_cast<const void*>(&wf_neeb), b_trace);
  uint32_t* more = nullptr;
  DG_CUDA(cudaMallocHost(&more, sizeof(uint32_t)));
  cudaEvent_t ev[6];
  for(auto& e : ev) { cudaEventCreate(&e); }
  for(int k = 0; k < 6; ++k) { ms[k] = 0.0; }
  wf_init<<<(std::max(tn.capacity, npix) + 255) / 256, 256, 0, st>>>(wf->dev, npix);
  bool ok = cudaGetLastError() == cudaSuccess;
  for(uint32_t wave = 0; ok && wave < wf->dev.max_waves + 1; ++wave) {
    cudaEventRecord(ev[0], st);
    wf_regen<<<g_regen, 256, 0, st>>>(sc, pp, wf->dev);
    cudaEventRecord(ev[1], st);
    wf_extend<<<g_ext, b_trace, 0, st>>>(sc, wf->dev);
    cudaEventRecord(ev[2], st);
    wf_shade<<<g_sha, b_shade, 0, st>>>(sc, pp, wf->dev);
    cudaEventRecord(ev[3], st);
    wf_shadow<<<g_shw, b_trace, 0, st>>>(sc, wf->dev);
    cudaEventRecord(ev[4], st);
    wf_neeb<<<g_nb, b_trace, 0, st>>>(sc, wf->dev);
    cudaEventRecord(ev[5], st);
    wf_control_host<<<1, 1, 0, st>>>(wf->dev, more);
    ok = cudaStreamSynchronize(st) == cudaSuccess;
    for(int k = 0; ok && k < 5; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      ms[k] += t;
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
  if(!ok) {
    return fail(DORT_ERR_CUDA, std::string("staged wavefront failed: ") +
                               cudaGetErrorString(cudaGetLastError()));
  }
  return DORT_OK;
}

int wavefront_counters(dort_scene* s, uint64_t* rays, uint32_t* waves, uint32_t* error,
                       cudaStream_t st) {
  if(!s->wavefront || !s->wavefront->mem) { return fail(DORT_ERR_INVALID, "no wavefront state"); }
  uint32_t c[C_COUNT];
  DG_CUDA(cudaMemcpyAsync(c, s->wavefront->dev.ctr, sizeof(c), cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaStreamSynchronize(st));
  *rays = uint64_t(c[C_RAYS_LO]) | (uint64_t(c[C_RAYS_LO + 1]) << 32);
  *waves = c[C_WAVES];
  *error = c[C_ERROR];
  return DORT_OK;
}

}  // namespace dort_gpu
