// Bidirectional path tracing: the "bdpt" renderer (BdptRenderer,
// bdpt_renderer.cpp:9-468).
//
// Per pixel sample: a light walk (random_light_walk, :96-180) and a camera
// walk (random_camera_walk, :182-290) with the forward and backward area pdfs
// of every vertex, then every pair (s light vertices, t camera vertices)
// within the depth limits is connected (path_contrib, :292-468) and weighted
// by the balance heuristic over the strategies that could have made the same
// path (path_weight, :470-678); t = 1 connections splat onto the film.  The
// walks are written through a vertex sink (a local array for the host check,
// device memory for the GPU's connection-parallel kernels in bdpt.cu), and
// one connection function serves both.
#pragma once
#include "lt.cuh"

namespace dort_gpu {

constexpr uint32_t kBdptVerts = 16;   // vertices per walk: max_depth <= 13

// The ray, surface, BSDF and light queries that the walks, the (s, t)
// connections and the MIS weight share.  When one kernel ran a whole sample,
// inlining them at every call site outgrew the SM's instruction cache (ncu:
// "no_instruction" the top stall at 48 cycles per issued instruction), and
// they were called out of line.  Each device kernel now runs one walk kind or
// one connection case, small enough to inline them: 148.8 against 136.5 M
// samples/s on the Cornell workload.  DORT_BD_NOINLINE keeps them out of
// line.
#ifdef DORT_BD_NOINLINE
#define DORT_BD_FN __host__ __device__ __noinline__
#else
#define DORT_BD_FN DG_HD
#endif
template<bool ANY_HIT, bool G>
DORT_BD_FN Hit bd_trace(const PtScene& sc, V3 o, float t_min, V3 d, float t_max) {
  return scene_trace<ANY_HIT, G>(sc, o, t_min, d, t_max);
}
template<bool G>
DORT_BD_FN bool bd_visible(const PtScene& sc, V3 a, float ea, V3 b, float eb) {
  return lt_visible<G>(sc, a, ea, b, eb);
}
template<bool G>
DORT_BD_FN SurfaceHit bd_surface(const PtScene& sc, const Hit& h, V3 o, V3 d) {
  return surface_at<G>(sc, h, o, d);
}
template<bool G>
DORT_BD_FN V3 bd_bsdf_eval(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo,
                                   uint32_t req) {
  return bsdf_eval<G>(m, fr, wi, wo, req);
}
template<bool G>
DORT_BD_FN float bd_bsdf_pdf(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo,
                                     uint32_t req) {
  return bsdf_pdf<G>(m, fr, wi, wo, req);
}
template<bool G>
DORT_BD_FN BsdfSample bd_bsdf_sample(const DevMaterial& m, const Frame& fr, V3 w,
                                             uint32_t req, float u, float v, float c) {
  return bsdf_sample<G>(m, fr, w, req, u, v, c);
}
template<bool G>
DORT_BD_FN LightSample bd_light_sample(const PtScene& sc, const DevLight& l, V3 p,
                                               float eps, float u, float v) {
  return light_sample<G>(sc, l, p, eps, u, v);
}

// Light flags (light.hpp:9-29).
enum : uint32_t {
  LF_DELTA_POS = 1, LF_DELTA_DIR = 2, LF_AREA = 4, LF_BACKGROUND = 8, LF_DISTANT = 16,
  LF_DELTA = LF_DELTA_POS | LF_DELTA_DIR
};

DG_HD uint32_t light_flags(const DevLight& l) {
  if(light_is_area(l)) { return LF_AREA; }
  if(l.kind == LIGHT_POINT) { return LF_DELTA_POS; }
  if(l.kind == LIGHT_DIR) { return LF_DELTA_DIR | LF_DISTANT; }
  return LF_BACKGROUND | LF_DISTANT;
}

// Light::ray_radiance_pdf (diffuse_light.cpp:95-103, point_light.cpp:48-52,
// directional_light.cpp:53-57, infinite_light.cpp:49-53,
// environment_light.cpp:79-83).
DG_HD float light_ray_pdf(const PtScene& sc, const DevLight& l, V3 dir, V3 nn) {
  float disk = kInvPi / sq(sc.radius);
  if(light_is_area(l)) { return dot(dir, nn) <= 0.f ? 0.f : (1.f / l.area) * kInvTwoPi; }
  if(l.kind == LIGHT_POINT) { return kInvFourPi; }
  if(l.kind == LIGHT_DIR) { return disk; }
  if(l.kind == LIGHT_INFINITE) { return disk * kInvFourPi; }
  return env_dir_pdf(sc.env, -dir) * disk;
}

// Camera::sample_ray_importance with its pdfs (pinhole_camera.cpp:13-31,
// thin_lens_camera.cpp:15-33, ortho_camera.cpp:13-26); returns the importance.
template<bool G>
DG_HD float camera_ray_importance(const PtParams& pp, uint32_t pixel, uint32_t sample, float fx,
                                  float fy, V3& o, V3& d, float& pos_pdf, float& dir_pdf) {
  camera_ray<G>(pp, pixel, sample, fx, fy, o, d);
  float area = image_plane_area(pp);
  if(G && pp.camera == CAMERA_ORTHO) {
    pos_pdf = 1.f / area;
    dir_pdf = 1.f;
    return 1.f / area;
  }
  V3 c = cam_local_vec(pp, d);
  float cos_t = c.z / length(c);
  dir_pdf = 1.f / (area * cos_t * cos_t * cos_t);
  if(G && pp.camera == CAMERA_THIN_LENS) {
    pos_pdf = kInvPi / sq(pp.lens_radius);
    return pos_pdf * dir_pdf;
  }
  pos_pdf = 1.f;
  return dir_pdf;
}

// Camera::ray_importance_pdf (pinhole_camera.cpp:84-100,
// thin_lens_camera.cpp:81-95, ortho_camera.cpp:61-63).
template<bool G>
DG_HD float camera_ray_pdf(const PtParams& pp, V3 origin, V3 wi) {
  float area = image_plane_area(pp);
  if(G && pp.camera == CAMERA_ORTHO) { return 1.f / area; }
  float fx, fy;
  if(G && pp.camera == CAMERA_THIN_LENS) {
    V3 lens = cam_local_point(pp, origin);
    V3 cw = cam_local_vec(pp, wi);
    if(!thin_film_pos(pp, lens, lens + cw, fx, fy)) { return 0.f; }
    float w = float(pp.width), h = float(pp.height);
    float k = pp.proj_dim / fmaxf(w, h);
    V3 focus = v3((fx - 0.5f * w) * k * pp.focal_distance, (fy - 0.5f * h) * k * pp.focal_distance,
                  pp.focal_distance);
    V3 seg = focus - lens;
    float cos_t = seg.z / length(seg);
    return kInvPi / (sq(pp.lens_radius) * area * cos_t * cos_t * cos_t);
  }
  V3 c = cam_local_vec(pp, wi);
  if(c.z <= 0.f) { return 0.f; }
  if(!plane_film_pos(pp, c.x / c.z, c.y / c.z, fx, fy)) { return 0.f; }
  float cos_t = c.z / length(c);
  return 1.f / (area * cos_t * cos_t * cos_t);
}

// Camera::pivot_importance_pdf (pinhole_camera.cpp:102-104,
// thin_lens_camera.cpp:97-99, ortho_camera.cpp:65-69).
template<bool G>
DG_HD float camera_pivot_pdf(const PtParams& pp, V3 p, V3 pivot) {
  if(G && pp.camera == CAMERA_THIN_LENS) { return kInvPi / sq(pp.lens_radius); }
  if(G && pp.camera == CAMERA_ORTHO) { return 1.f / length_sq(p - pivot); }
  return 1.f;
}

struct BVert {
  V3 p;
  float eps;
  V3 nn;            // geometric (= shading) normal; the ray direction at z0
  V3 s;             // BSDF frame tangent (frame = s, cross(nn, s), nn)
  V3 alpha;
  float fwd_pdf, bwd_pdf;
  uint32_t mat;     // material index + 1, 0: no BSDF
  uint32_t prim;    // hit primitive (per-triangle albedo)
  uint32_t light;   // area light index + 1 hit by the camera walk, 0 if none
  uint32_t bg;      // background light index + 1 of a virtual vertex, 0 if none
  uint32_t delta;   // the vertex was sampled with a delta BxDF
};

DG_HD Frame bvert_frame(const BVert& v) {
  Frame f;
  f.n = v.nn;
  f.s = v.s;
  f.t = cross(v.nn, v.s);
  return f;
}

DG_HD DevMaterial bvert_material(const PtScene& sc, const BVert& v) {
  SurfaceHit g;
  g.mat = v.mat - 1u;
  g.tri = v.prim;
  return material_at(sc, g);
}

DG_HD BVert bvert_surface(const SurfaceHit& g) {
  BVert v;
  v.p = g.p;
  v.eps = g.eps;
  v.nn = g.n;
  v.s = g.frame.s;
  v.alpha = v3(0.f, 0.f, 0.f);
  v.fwd_pdf = 0.f;
  v.bwd_pdf = 0.f;
  v.mat = g.mat + 1u;
  v.prim = g.tri;
  v.light = 0;
  v.bg = 0;
  v.delta = 0;
  return v;
}

DG_HD BVert bvert_empty() {
  BVert v;
  v.p = v3(0.f, 0.f, 0.f);
  v.eps = 0.f;
  v.nn = v3(0.f, 0.f, 0.f);
  v.s = v3(0.f, 0.f, 0.f);
  v.alpha = v3(0.f, 0.f, 0.f);
  v.fwd_pdf = 0.f;
  v.bwd_pdf = 0.f;
  v.mat = v.prim = v.light = v.bg = v.delta = 0;
  return v;
}

// Where a walk's vertices live.
//   LocalWalk  an array of one sample's vertices (the host check).
//   SoaWalk    the device's connection-parallel form: vertex k of sample i of
//              a chunk as five float4 words, word w at (5 k + w) * stride + i,
//              so that the lanes of a warp (consecutive samples) store and
//              load whole lines.  get() reads through the read-only path: a
//              walk is read only by launches after the one that wrote it.
struct LocalWalk {
  BVert* v;
  DG_HD void put(uint32_t k, const BVert& x) const { v[k] = x; }
  DG_HD BVert get(uint32_t k) const { return v[k]; }
};

struct SoaWalk {
  float4* base;
  uint32_t stride, i;
  DG_HD void put(uint32_t k, const BVert& x) const {
    float4* q = base + size_t(5 * k) * stride + i;
    const size_t st = stride;
    q[0] = make_float4(x.p.x, x.p.y, x.p.z, x.eps);
    q[st] = make_float4(x.nn.x, x.nn.y, x.nn.z, x.fwd_pdf);
    q[2 * st] = make_float4(x.s.x, x.s.y, x.s.z, x.bwd_pdf);
    q[3 * st] = make_float4(x.alpha.x, x.alpha.y, x.alpha.z, DG_AS_FLOAT(x.mat));
    q[4 * st] = make_float4(DG_AS_FLOAT(x.prim), DG_AS_FLOAT(x.light), DG_AS_FLOAT(x.bg),
                            DG_AS_FLOAT(x.delta));
  }
  DG_HD BVert get(uint32_t k) const {
    const float4* q = base + size_t(5 * k) * stride + i;
    const size_t st = stride;
    float4 a = DG_LDG(q), b = DG_LDG(q + st), c = DG_LDG(q + 2 * st);
    float4 d = DG_LDG(q + 3 * st), e = DG_LDG(q + 4 * st);
    BVert v;
    v.p = v3(a.x, a.y, a.z);
    v.eps = a.w;
    v.nn = v3(b.x, b.y, b.z);
    v.fwd_pdf = b.w;
    v.s = v3(c.x, c.y, c.z);
    v.bwd_pdf = c.w;
    v.alpha = v3(d.x, d.y, d.z);
    v.mat = DG_AS_UINT(d.w);
    v.prim = DG_AS_UINT(e.x);
    v.light = DG_AS_UINT(e.y);
    v.bg = DG_AS_UINT(e.z);
    v.delta = DG_AS_UINT(e.w);
    return v;
  }
};

// Dimension blocks of one BDPT sample:
//   0                 film jitter (a, b); the thin lens's lens point (c, d)
//   1, 2              light pick, light ray position and direction
//   16 + 2k, 17 + 2k  light walk bounce k: BSDF uv, component, roulette
//   64 + 2k, 65 + 2k  camera walk bounce k: BSDF uv, component, roulette,
//                     background light pick
//   256 + 32 s + t    the connection (s, t): light / camera samples
constexpr uint32_t kBdLightWalk = 16, kBdCameraWalk = 64, kBdConnect = 256;

struct BdptCtx {
  const PtScene& sc;
  const PtParams& pp;
  uint32_t pixel, sample;
};

// random_light_walk (bdpt_renderer.cpp:96-180); returns the vertex count.
// The walk's last vertex stays in registers until the next one is made (it
// receives its backward pdf then), so every vertex is stored once.
template<bool G, class W>
DG_HD uint32_t bdpt_light_walk(const BdptCtx& c, uint32_t light_i, float pick, const W& lw,
                               uint32_t& rays) {
  const PtScene& sc = c.sc;
  const DevLight& l = sc.lights[light_i];
  Rand4 r1 = rand4(c.pp.seed, c.pixel, c.sample, 1);
  Rand4 r2 = rand4(c.pp.seed, c.pixel, c.sample, 2);
  LightRay ray;
  if(!light_sample_ray<G>(sc, l, r1.b, r1.c, r1.d, r2.a, ray)) { return 0; }
  if(ray.pos_pdf == 0.f || ray.dir_pdf == 0.f) { return 0; }
  const bool distant = (light_flags(l) & LF_DISTANT) != 0;
  BVert prev = bvert_empty();
  prev.p = ray.o;
  prev.eps = ray.eps;
  prev.nn = ray.nn;
  prev.fwd_pdf = ray.pos_pdf;
  prev.alpha = ray.L * (1.f / (ray.pos_pdf * pick));
  uint32_t n = 1;
  V3 prev_f = v3(1.f, 1.f, 1.f);
  float fwd_dir_pdf = ray.dir_pdf;
  V3 o = ray.o, d = ray.d;
  float eps = ray.eps;
  for(uint32_t b = 0; b <= c.pp.max_depth && n < kBdptVerts; ++b) {
    ++rays;
    Hit h = bd_trace<false, G>(sc, o, eps, d, INFINITY);
    if(h.prim == kMiss) { break; }
    SurfaceHit g = bd_surface<G>(sc, h, o, d);
    DevMaterial m = material_at(sc, g);
    V3 wi = -d;
    Rand4 ra = rand4(c.pp.seed, c.pixel, c.sample, kBdLightWalk + 2 * b);
    // Bsdf::sample_camera_f: the same sampling from either side here
    BsdfSample bs = bd_bsdf_sample<G>(m, g.frame, wi, F_ALL, ra.a, ra.b, ra.c);
    if(bs.pdf == 0.f) { break; }
    V3 wo = normalize(bs.w);
    float bwd_dir_pdf = bd_bsdf_pdf<G>(m, g.frame, wi, wo, F_ALL);   // light_f_pdf(wi, wo)
    float dist2 = length_sq(g.p - prev.p);
    if(dist2 < 1e-9f) { break; }
    V3 scale = prev_f * (fabsf(dot(prev.nn, wi)) / fwd_dir_pdf);
    if(b >= 2) {
      float rr = fminf(average(scale), 0.9f);
      if(ra.d > rr) { break; }
      scale = scale * (1.f / rr);
    }
    BVert y = bvert_surface(g);
    y.fwd_pdf = (b == 0 && distant) ? ray.dir_pdf : fwd_dir_pdf * fabsf(dot(y.nn, wi)) / dist2;
    y.alpha = prev.alpha * scale;
    y.delta = (bs.flags & F_DELTA) ? 1u : 0u;
    if(is_black(y.alpha)) { break; }
    prev.bwd_pdf = bwd_dir_pdf * fabsf(dot(prev.nn, wi)) / dist2;
    lw.put(n - 1, prev);
    prev = y;
    ++n;
    prev_f = bs.f;
    fwd_dir_pdf = bs.pdf;
    o = y.p;
    d = wo;
    eps = g.eps;
  }
  lw.put(n - 1, prev);
  return n;
}

// random_camera_walk (bdpt_renderer.cpp:182-290); returns the vertex count.
// `emit` collects bit k for a vertex k that is emissive (an area light hit)
// and bit 16 + k for a virtual background vertex.
template<bool G, class W>
DG_HD uint32_t bdpt_camera_walk(const BdptCtx& c, float fx, float fy, const W& cw,
                                uint32_t& rays, uint32_t& emit) {
  const PtScene& sc = c.sc;
  emit = 0;
  V3 o, d;
  float pos_pdf, dir_pdf;
  float We = camera_ray_importance<G>(c.pp, c.pixel, c.sample, fx, fy, o, d, pos_pdf, dir_pdf);
  if(pos_pdf == 0.f || dir_pdf == 0.f) { return 0; }
  BVert prev = bvert_empty();
  prev.p = o;
  prev.nn = d;
  prev.fwd_pdf = pos_pdf;
  prev.alpha = v3(We, We, We) * (1.f / pos_pdf);
  uint32_t n = 1;
  V3 prev_f = v3(1.f, 1.f, 1.f);
  float fwd_dir_pdf = dir_pdf;
  float eps = 0.f;
  for(uint32_t b = 0; b <= c.pp.max_depth && n < kBdptVerts; ++b) {
    if(is_black(prev.alpha)) { break; }
    Rand4 ra = rand4(c.pp.seed, c.pixel, c.sample, kBdCameraWalk + 2 * b);
    Rand4 rb = rand4(c.pp.seed, c.pixel, c.sample, kBdCameraWalk + 2 * b + 1);
    V3 scale = prev_f * (fabsf(dot(prev.nn, d)) / fwd_dir_pdf);
    if(b >= 2) {
      float rr = fminf(average(scale), 0.9f);
      if(ra.d > rr) { break; }
      scale = scale * (1.f / rr);
    }
    ++rays;
    Hit h = bd_trace<false, G>(sc, o, eps, d, INFINITY);
    if(h.prim == kMiss) {
      // a virtual vertex on the background light picked by power
      // (background_light_distrib)
      if(sc.bg_count == 0) { break; }
      float p0 = distrib_pdf(sc.light_cdf, sc.light_count + 1, sc.bg_light[0]);
      float p1 = sc.bg_count > 1 ? distrib_pdf(sc.light_cdf, sc.light_count + 1, sc.bg_light[1])
                                 : 0.f;
      float tot = p0 + p1;
      if(!(tot > 0.f)) { break; }
      uint32_t k = (sc.bg_count > 1 && rb.a * tot >= p0) ? 1u : 0u;
      float bg_pdf = (k == 0 ? p0 : p1) / tot;
      if(bg_pdf == 0.f) { break; }
      BVert zb = bvert_empty();
      zb.p = prev.p + d;
      zb.bg = sc.bg_light[k] + 1u;
      zb.fwd_pdf = fwd_dir_pdf;
      zb.alpha = prev.alpha * scale * (1.f / bg_pdf);
      cw.put(n - 1, prev);
      prev = zb;
      emit |= 1u << (16 + n);
      ++n;
      break;
    }
    SurfaceHit g = bd_surface<G>(sc, h, o, d);
    DevMaterial m = material_at(sc, g);
    V3 wo = -d;
    BsdfSample bs = bd_bsdf_sample<G>(m, g.frame, wo, F_ALL, ra.a, ra.b, ra.c);
    float dist2 = length_sq(g.p - prev.p);
    if(dist2 < 1e-9f) { break; }
    BVert z = bvert_surface(g);
    z.light = g.light;
    z.fwd_pdf = fwd_dir_pdf * fabsf(dot(z.nn, wo)) / dist2;
    z.alpha = prev.alpha * scale;
    z.delta = (bs.flags & F_DELTA) ? 1u : 0u;
    if(is_black(z.alpha) && z.light == 0) { break; }
    if(z.light != 0) { emit |= 1u << n; }
    if(bs.pdf == 0.f) {
      prev.bwd_pdf = 0.f;
      cw.put(n - 1, prev);
      prev = z;
      ++n;
      break;
    }
    V3 wi = normalize(bs.w);
    float bwd_dir_pdf = bd_bsdf_pdf<G>(m, g.frame, wo, wi, F_ALL);   // camera_f_pdf(wo, wi)
    prev.bwd_pdf = bwd_dir_pdf * fabsf(dot(prev.nn, wo)) / dist2;
    cw.put(n - 1, prev);
    prev = z;
    ++n;
    prev_f = bs.f;
    fwd_dir_pdf = bs.pdf;
    o = z.p;
    d = wi;
    eps = g.eps;
  }
  cw.put(n - 1, prev);
  return n;
}

// The path of s light and t camera vertices, as path_weight indexes it:
// x[0 .. s-1] = light vertices, x[s .. s+t-1] = camera vertices in reverse.
// A connection that makes its own end vertex (s = 1: a new light sample;
// t = 1: a new camera point) puts it in place of the walk's first one.
template<class W>
struct BdptPath {
  W lw, cw;
  const BVert* first_light;    // replaces light vertex 0 if set
  const BVert* first_camera;   // replaces camera vertex 0 if set
  uint32_t s, t;
  DG_HD BVert light_at(uint32_t i) const {
    return (i == 0 && first_light) ? *first_light : lw.get(i);
  }
  DG_HD BVert camera_at(uint32_t i) const {
    return (i == 0 && first_camera) ? *first_camera : cw.get(i);
  }
  DG_HD BVert at(uint32_t i) const {
    return i < s ? light_at(i) : camera_at(t - (i - s + 1));
  }
};

// path_weight (bdpt_renderer.cpp:470-678): the balance heuristic over the
// strategies (s', t') with s' + t' = s + t.
template<bool G, class P>
DG_HD float bdpt_weight(const BdptCtx& c, const DevLight& light, const P& x) {
  const PtScene& sc = c.sc;
  const PtParams& pp = c.pp;
  const uint32_t s = x.s, t = x.t;
  const uint32_t lf = light_flags(light);
  if(x.camera_at(t - 1).bg != 0 && s != 0) { return 0.f; }
  if(s + t == 2) {
    if(lf & (LF_AREA | LF_BACKGROUND)) { return s == 0 ? 1.f : 0.f; }
    return t == 1 ? 1.f : 0.f;
  }
  float x0_pivot_pdf;
  if(s == 1) {
    x0_pivot_pdf = x.at(0).fwd_pdf;
  } else {
    const BVert& x0 = x.at(0);
    const BVert& x1 = x.at(1);
    V3 wi = normalize(x0.p - x1.p);
    float dir_pdf = light_pivot_pdf<G>(sc, light, wi, x1.p);
    x0_pivot_pdf = (lf & LF_DISTANT) ? dir_pdf
                                     : dir_pdf * fabsf(dot(x0.nn, wi)) / length_sq(x0.p - x1.p);
  }

  auto pdf_light = [&](uint32_t i) -> float {
    if(i == 0) { return x0_pivot_pdf; }
    if(i == 1) {
      if(x0_pivot_pdf == 0.f) { return 0.f; }
      const BVert& x0 = x.at(0);
      const BVert& x1 = x.at(1);
      V3 wi = normalize(x0.p - x1.p);
      float ray_pdf;
      if(s >= 2) {
        if(lf & LF_DISTANT) {
          ray_pdf = x1.fwd_pdf * (x0.fwd_pdf * fabsf(dot(wi, x1.nn)));
        } else {
          ray_pdf = x0.fwd_pdf * x1.fwd_pdf;
        }
      } else {
        float ang = light_ray_pdf(sc, light, -wi, x0.nn);
        ray_pdf = (lf & LF_DISTANT) ? ang * fabsf(dot(x1.nn, wi))
                                    : ang * fabsf(dot(x1.nn, wi)) / length_sq(x0.p - x1.p);
      }
      return ray_pdf / x0_pivot_pdf;
    }
    if(i < s) { return x.at(i).fwd_pdf; }
    if(i == s && t != 1) {
      const BVert& xo = x.at(i);
      const BVert& xm = x.at(i - 1);
      const BVert& xi = x.at(i - 2);
      V3 bwi = normalize(xi.p - xm.p), bwo = normalize(xo.p - xm.p);
      DevMaterial m = bvert_material(sc, xm);
      float dir_pdf = bd_bsdf_pdf<G>(m, bvert_frame(xm), bwo, bwi, F_ALL);   // camera_f_pdf
      float d2 = length_sq(xo.p - xm.p);
      if(d2 == 0.f) { return 0.f; }
      return dir_pdf * fabsf(dot(bwo, xo.nn)) / d2;
    }
    return x.at(i).bwd_pdf;    // i > s, i < s + t - 1
  };

  auto pdf_camera = [&](uint32_t i) -> float {
    if(i == s + t - 2) {
      const BVert& z1 = x.at(s + t - 2);
      const BVert& z0 = x.at(s + t - 1);
      V3 wi = normalize(z1.p - z0.p);
      float ray_area_pdf;
      if(t >= 2) {
        ray_area_pdf = z0.fwd_pdf * z1.fwd_pdf;
      } else {
        float rp = camera_ray_pdf<G>(pp, z0.p, wi);
        ray_area_pdf = rp * fabsf(dot(wi, z1.nn)) / length_sq(z1.p - z0.p);
      }
      float pivot_area_pdf = t == 1 ? z0.fwd_pdf : camera_pivot_pdf<G>(pp, z0.p, z1.p);
      if(pivot_area_pdf == 0.f) { return 0.f; }
      return ray_area_pdf / pivot_area_pdf;
    }
    if(i < s + t - 2 && i >= s) { return x.at(i).fwd_pdf; }
    if(i == s - 1 && t >= 2) {
      if(i == 0 && (lf & LF_DELTA)) { return 0.f; }
      const BVert& xi = x.at(i);
      const BVert& xm = x.at(i + 1);
      const BVert& xo = x.at(i + 2);
      V3 bwi = normalize(xi.p - xm.p), bwo = normalize(xo.p - xm.p);
      DevMaterial m = bvert_material(sc, xm);
      float dir_pdf = bd_bsdf_pdf<G>(m, bvert_frame(xm), bwi, bwo, F_ALL);   // light_f_pdf
      if(i == 0 && (lf & LF_DISTANT)) { return dir_pdf; }
      return dir_pdf * fabsf(dot(xi.nn, bwi)) / length_sq(xi.p - xm.p);
    }
    return x.at(i).bwd_pdf;    // i < s - 1
  };

  float inv_sum = 1.f;
  float r = 1.f;
  for(uint32_t j = 1; j <= t - 1; ++j) {
    float fp = pdf_light(s + j - 1);
    float bp = pdf_camera(s + j - 1);
    if(bp == 0.f) { break; }
    r *= fp / bp;
    if(r == 0.f) { break; }
    if(x.at(s + j - 1).delta) { continue; }
    if(s + j < s + t && x.at(s + j).delta) { continue; }
    inv_sum += r;
  }
  r = 1.f;
  for(uint32_t j = 1; j <= s; ++j) {
    if(s - j == 0 && (lf & LF_DELTA)) { break; }
    float fp = pdf_camera(s - j);
    float bp = pdf_light(s - j);
    if(bp == 0.f) { break; }
    r *= fp / bp;
    if(r == 0.f) { break; }
    if(x.at(s - j).delta) { continue; }
    if(j < s && x.at(s - j - 1).delta) { continue; }
    inv_sum += r;
  }
  return 1.f / inv_sum;
}

// One sample's data beside its walks: vertex counts, the light picked for
// the light walk with its probability, the film position.
struct BdptSampleData {
  uint32_t ns, nt, light_i;
  float pick, fx, fy;
};

// Connection cases, by the code each runs (the branches of sample_path's
// connection loop, bdpt_renderer.cpp:292-468):
//   kBdCaseS0  s = 0: the camera walk's vertex t - 1 is emissive (no ray)
//   kBdCaseS1  s = 1, t >= 2: a new light sample seen from camera vertex t - 1
//   kBdCaseT1  t = 1: a new camera point seen from light vertex s - 1 (a
//              film splat)
//   kBdCaseST  s >= 2, t >= 2: the two walks' end vertices joined
// kBdCaseAll compiles every branch (the host's loop over one sample).
enum : uint32_t {
  kBdCaseS0 = 0, kBdCaseS1 = 1, kBdCaseT1 = 2, kBdCaseST = 3, kBdCases = 4, kBdCaseAll = 4
};

// The case of connection (s, t), or kBdCases when the loop skips it before
// drawing its random numbers or always rejects it: `emit` is the camera
// walk's mask (bdpt_camera_walk).
DG_HD uint32_t bdpt_pair_case(const PtParams& pp, bool use_t1, uint32_t emit, uint32_t s,
                              uint32_t t) {
  if(t == 1 && !use_t1) { return kBdCases; }
  if(s + t < pp.min_depth + 2 || s + t > pp.max_depth + 2) { return kBdCases; }
  const bool bg = (emit >> (16 + t - 1)) & 1u, light = (emit >> (t - 1)) & 1u;
  if(s > 0 && bg) { return kBdCases; }
  if(s == 0) { return (bg || light) ? kBdCaseS0 : kBdCases; }   // t >= 2 as s + t >= 2
  if(t == 1) { return kBdCaseT1; }
  return s == 1 ? kBdCaseS1 : kBdCaseST;
}

// One connection (s, t) of a sample: false if it adds nothing, else its
// weighted contribution `wc` and, for t = 1, the film position it splats to.
// The body of sample_path's connection loop (bdpt_renderer.cpp:292-468).
template<bool G, uint32_t CASE, class W>
DG_HD bool bdpt_connect(const BdptCtx& c, const W& lw, const W& cw, const BdptSampleData& sd,
                        uint32_t s, uint32_t t, V3& wc, float& sfx, float& sfy, uint32_t& rays) {
  constexpr bool kAll = CASE == kBdCaseAll;
  const PtScene& sc = c.sc;
  const PtParams& pp = c.pp;
  const uint32_t light_i = sd.light_i;
  Rand4 rc = rand4(pp.seed, c.pixel, c.sample, kBdConnect + 32 * s + t);
  const BVert last_camera = cw.get(t - 1);
  uint32_t new_light = light_i;
  // the connection's own end vertices where it makes new ones (s = 1 light
  // sample, t = 1 camera point), else the walks' first vertices
  BVert first_light, first_camera;
  const BVert* fl = nullptr;
  const BVert* fc = nullptr;
  sfx = sd.fx;
  sfy = sd.fy;
  V3 contrib = v3(0.f, 0.f, 0.f);
  if(s > 0 && last_camera.bg != 0) {
    return false;
  } else if(s == 1 && t == 1) {
    if constexpr(kAll || CASE == kBdCaseT1) {
      if(G && pp.camera == CAMERA_ORTHO) { return false; }   // CAMERA_DIR_BY_POS_DELTA
      float cam_pdf;
      V3 cp = camera_sample_point<G>(pp, rc.a, rc.b, cam_pdf);
      if(cam_pdf == 0.f) { return false; }
      LightSample ls = bd_light_sample<G>(sc, sc.lights[light_i], cp, 0.f, rc.c, rc.d);
      if(ls.pdf == 0.f || is_black(ls.L)) { return false; }
      float We = camera_eval_importance<G>(pp, cp, ls.wi, sfx, sfy);
      if(We == 0.f) { return false; }
      if(sd.pick == 0.f) { return false; }
      ++rays;
      Hit h = bd_trace<true, G>(sc, ls.o, ls.tmin, ls.d, ls.tmax);
      if(h.prim != kMiss) { return false; }
      contrib = ls.L * (We / (cam_pdf * ls.pdf * sd.pick));
    } else {
      return false;
    }
  } else if(s == 0) {
    if constexpr(kAll || CASE == kBdCaseS0) {
      const BVert prev_camera = cw.get(t - 2);
      if(last_camera.bg != 0) {
        const DevLight& bl = sc.lights[last_camera.bg - 1u];
        V3 Le = background_radiance(sc, bl, normalize(last_camera.p - prev_camera.p));
        if(is_black(Le)) { return false; }
        new_light = last_camera.bg - 1u;
        contrib = Le * last_camera.alpha;
      } else if(last_camera.light != 0) {
        const DevLight& al = sc.lights[last_camera.light - 1u];
        V3 Le = area_eval_radiance(sc, al, last_camera.p, last_camera.nn, prev_camera.p);
        if(is_black(Le)) { return false; }
        new_light = last_camera.light - 1u;
        contrib = Le * last_camera.alpha;
      } else {
        return false;
      }
    } else {
      return false;
    }
  } else if(s == 1) {
    if constexpr(kAll || CASE == kBdCaseS1) {
      uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, rc.a);
      float lp = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
      new_light = li;
      if(lp == 0.f) { return false; }
      const DevLight& l2 = sc.lights[li];
      LightSample ls = bd_light_sample<G>(sc, l2, last_camera.p, last_camera.eps, rc.b, rc.c);
      if(is_black(ls.L) || ls.pdf == 0.f) { return false; }
      ++rays;
      Hit h = bd_trace<true, G>(sc, ls.o, ls.tmin, ls.d, ls.tmax);
      if(h.prim != kMiss) { return false; }
      V3 bwo = normalize(cw.get(t - 2).p - last_camera.p);
      DevMaterial m = bvert_material(sc, last_camera);
      Frame fr = bvert_frame(last_camera);
      V3 f = bd_bsdf_eval<G>(m, fr, ls.wi, bwo, F_ALL);
      if(is_black(f)) { return false; }
      first_light = bvert_empty();
      if(light_flags(l2) & LF_DISTANT) {
        first_light.p = last_camera.p + ls.wi;
        first_light.fwd_pdf = ls.pdf;
      } else {
        first_light.p = ls.p;
        first_light.eps = ls.p_eps;
        first_light.nn = ls.nn;
        first_light.fwd_pdf = ls.pdf * fabsf(dot(ls.nn, ls.wi)) / length_sq(ls.p - last_camera.p);
      }
      first_light.delta = (light_flags(l2) & LF_DELTA_DIR) ? 1u : 0u;
      first_light.bwd_pdf = bd_bsdf_pdf<G>(m, fr, ls.wi, bwo, F_ALL);
      fl = &first_light;
      contrib = last_camera.alpha * f * ls.L *
                (fabsf(dot(last_camera.nn, ls.wi)) / (lp * ls.pdf));
    } else {
      return false;
    }
  } else if(t == 1) {
    if constexpr(kAll || CASE == kBdCaseT1) {
      const BVert last_light = lw.get(s - 1);
      CameraPivot cam;
      if(!camera_pivot_importance<G>(pp, last_light.p, rc.a, rc.b, cam) || cam.We == 0.f ||
         cam.pdf == 0.f) {
        return false;
      }
      sfx = cam.fx;
      sfy = cam.fy;
      V3 wi = normalize(lw.get(s - 2).p - last_light.p);
      V3 wo = normalize(cam.p - last_light.p);
      DevMaterial m = bvert_material(sc, last_light);
      V3 f = bd_bsdf_eval<G>(m, bvert_frame(last_light), wi, wo, F_ALL);
      if(is_black(f)) { return false; }
      ++rays;
      if(!bd_visible<G>(sc, last_light.p, last_light.eps, cam.p, 0.f)) { return false; }
      first_camera = bvert_empty();
      first_camera.p = cam.p;
      first_camera.fwd_pdf = cam.pdf;
      first_camera.alpha = v3(cam.We, cam.We, cam.We);
      fc = &first_camera;
      contrib = last_light.alpha * f *
                (cam.We * fabsf(dot(last_light.nn, wo)) /
                 (length_sq(cam.p - last_light.p) * cam.pdf));
    } else {
      return false;
    }
  } else {
    // s >= 2 && t >= 2
    if constexpr(kAll || CASE == kBdCaseST) {
      const BVert last_light = lw.get(s - 1);
      ++rays;
      if(!bd_visible<G>(sc, last_light.p, last_light.eps, last_camera.p, last_camera.eps)) {
        return false;
      }
      V3 lwi = normalize(lw.get(s - 2).p - last_light.p);
      V3 cwo = normalize(cw.get(t - 2).p - last_camera.p);
      V3 wo = normalize(last_camera.p - last_light.p);
      DevMaterial ml = bvert_material(sc, last_light);
      V3 fl3 = bd_bsdf_eval<G>(ml, bvert_frame(last_light), lwi, wo, F_ALL);
      if(is_black(fl3)) { return false; }
      DevMaterial mc = bvert_material(sc, last_camera);
      V3 fc3 = bd_bsdf_eval<G>(mc, bvert_frame(last_camera), -wo, cwo, F_ALL);
      if(is_black(fc3)) { return false; }
      float geom = fabsf(dot(wo, last_light.nn)) * fabsf(dot(wo, last_camera.nn)) /
                   length_sq(last_light.p - last_camera.p);
      contrib = last_light.alpha * last_camera.alpha * fl3 * fc3 * geom;
    } else {
      return false;
    }
  }
  if(is_black(contrib)) { return false; }
  BdptPath<W> path{lw, cw, fl, fc, s, t};
  float w = bdpt_weight<G>(c, sc.lights[new_light], path);
  wc = contrib * w;
  return true;
}

// One pixel sample (sample_path, bdpt_renderer.cpp:40-94) in one thread, as
// the host check runs it: the camera-side value is returned, t = 1 splats go
// straight to the film.  The device runs the same walks and connections
// spread over kernels (bdpt.cu).
template<bool G>
DG_HD V3 bdpt_sample(const PtScene& sc, const PtParams& pp, uint32_t pixel, uint32_t sample,
                     float fx, float fy, bool use_t1, float* splat, uint32_t& rays) {
  V3 total = v3(0.f, 0.f, 0.f);
  if(sc.light_count == 0) { return total; }
  BdptCtx c{sc, pp, pixel, sample};
  Rand4 r1 = rand4(pp.seed, pixel, sample, 1);
  uint32_t light_i = distrib_sample(sc.light_cdf, sc.light_count + 1, r1.a);
  float pick = distrib_pdf(sc.light_cdf, sc.light_count + 1, light_i);
  BVert lwa[kBdptVerts], cwa[kBdptVerts];
  const LocalWalk lw{lwa}, cw{cwa};
  uint32_t emit = 0;
  uint32_t ns = pick > 0.f ? bdpt_light_walk<G>(c, light_i, pick, lw, rays) : 0u;
  uint32_t nt = bdpt_camera_walk<G>(c, fx, fy, cw, rays, emit);
  if(ns == 0) { lwa[0] = bvert_empty(); }
  if(nt == 0) { return total; }
  const BdptSampleData sd{ns, nt, light_i, pick, fx, fy};
  for(uint32_t s = 0; s <= ns; ++s) {
    for(uint32_t t = 1; t <= nt; ++t) {
      if(bdpt_pair_case(pp, use_t1, emit, s, t) == kBdCases) { continue; }
      V3 wc;
      float sfx, sfy;
      if(!bdpt_connect<G, kBdCaseAll>(c, lw, cw, sd, s, t, wc, sfx, sfy, rays)) { continue; }
      if(t == 1) {
        lt_splat(splat, pp, sfx, sfy, wc);
      } else {
        total = total + wc;
      }
    }
  }
  return total;
}

}  // namespace dort_gpu
