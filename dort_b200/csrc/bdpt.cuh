// Bidirectional path tracing: the "bdpt" renderer (BdptRenderer,
// bdpt_renderer.cpp:9-468).
//
// Per pixel sample: a light walk (random_light_walk, :96-180) and a camera
// walk (random_camera_walk, :182-290) with the forward and backward area pdfs
// of every vertex, then every pair (s light vertices, t camera vertices)
// within the depth limits is connected (path_contrib, :292-468) and weighted
// by the balance heuristic over the strategies that could have made the same
// path (path_weight, :470-678); t = 1 connections splat onto the film.  The
// walks live in local arrays of kBdptVerts vertices.
#pragma once
#include "lt.cuh"

namespace dort_gpu {

constexpr uint32_t kBdptVerts = 16;   // vertices per walk: max_depth <= 13

// Out-of-line entry points for the ray, surface, BSDF and light queries
// that the walks, the (s, t) connections and the MIS weight share.  Each is
// called from several places of one sample; inlined at every call site, the
// kernel's code outgrew the SM's instruction cache (ncu on the Cornell
// workload: "no_instruction" the top stall at 48 cycles per issued
// instruction, 7 % of issue slots busy).  One copy of each, reached by a
// call, keeps the loop's code small.
template<bool ANY_HIT, bool G>
DG_HD __noinline__ Hit bd_trace(const PtScene& sc, V3 o, float t_min, V3 d, float t_max) {
  return scene_trace<ANY_HIT, G>(sc, o, t_min, d, t_max);
}
template<bool G>
DG_HD __noinline__ bool bd_visible(const PtScene& sc, V3 a, float ea, V3 b, float eb) {
  return lt_visible<G>(sc, a, ea, b, eb);
}
template<bool G>
DG_HD __noinline__ SurfaceHit bd_surface(const PtScene& sc, const Hit& h, V3 o, V3 d) {
  return surface_at<G>(sc, h, o, d);
}
template<bool G>
DG_HD __noinline__ V3 bd_bsdf_eval(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo,
                                   uint32_t req) {
  return bsdf_eval<G>(m, fr, wi, wo, req);
}
template<bool G>
DG_HD __noinline__ float bd_bsdf_pdf(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo,
                                     uint32_t req) {
  return bsdf_pdf<G>(m, fr, wi, wo, req);
}
template<bool G>
DG_HD __noinline__ BsdfSample bd_bsdf_sample(const DevMaterial& m, const Frame& fr, V3 w,
                                             uint32_t req, float u, float v, float c) {
  return bsdf_sample<G>(m, fr, w, req, u, v, c);
}
template<bool G>
DG_HD __noinline__ LightSample bd_light_sample(const PtScene& sc, const DevLight& l, V3 p,
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
template<bool G>
DG_HD uint32_t bdpt_light_walk(const BdptCtx& c, uint32_t light_i, float pick, BVert* lw,
                               uint32_t& rays) {
  const PtScene& sc = c.sc;
  const DevLight& l = sc.lights[light_i];
  Rand4 r1 = rand4(c.pp.seed, c.pixel, c.sample, 1);
  Rand4 r2 = rand4(c.pp.seed, c.pixel, c.sample, 2);
  LightRay ray;
  if(!light_sample_ray<G>(sc, l, r1.b, r1.c, r1.d, r2.a, ray)) { return 0; }
  if(ray.pos_pdf == 0.f || ray.dir_pdf == 0.f) { return 0; }
  const bool distant = (light_flags(l) & LF_DISTANT) != 0;
  BVert y0 = bvert_empty();
  y0.p = ray.o;
  y0.eps = ray.eps;
  y0.nn = ray.nn;
  y0.fwd_pdf = ray.pos_pdf;
  y0.alpha = ray.L * (1.f / (ray.pos_pdf * pick));
  lw[0] = y0;
  uint32_t n = 1;
  V3 prev_f = v3(1.f, 1.f, 1.f);
  float fwd_dir_pdf = ray.dir_pdf;
  V3 o = ray.o, d = ray.d;
  float eps = ray.eps;
  for(uint32_t b = 0; b <= c.pp.max_depth && n < kBdptVerts; ++b) {
    BVert& prev = lw[n - 1];
    ++rays;
    Hit h = bd_trace<false, G>(sc, o, eps, d, INFINITY);
    if(h.prim == kMiss) { break; }
    SurfaceHit g = bd_surface<G>(sc, h, o, d);
    DevMaterial m = material_at(sc, g);
    V3 wi = -d;
    Rand4 ra = rand4(c.pp.seed, c.pixel, c.sample, kBdLightWalk + 2 * b);
    Rand4 rb = rand4(c.pp.seed, c.pixel, c.sample, kBdLightWalk + 2 * b + 1);
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
    prev_f = bs.f;
    fwd_dir_pdf = bs.pdf;
    o = y.p;
    d = wo;
    eps = g.eps;
    lw[n++] = y;
    (void)rb;
  }
  return n;
}

// random_camera_walk (bdpt_renderer.cpp:182-290); returns the vertex count.
template<bool G>
DG_HD uint32_t bdpt_camera_walk(const BdptCtx& c, float fx, float fy, BVert* cw,
                                uint32_t& rays) {
  const PtScene& sc = c.sc;
  V3 o, d;
  float pos_pdf, dir_pdf;
  float We = camera_ray_importance<G>(c.pp, c.pixel, c.sample, fx, fy, o, d, pos_pdf, dir_pdf);
  if(pos_pdf == 0.f || dir_pdf == 0.f) { return 0; }
  BVert z0 = bvert_empty();
  z0.p = o;
  z0.nn = d;
  z0.fwd_pdf = pos_pdf;
  z0.alpha = v3(We, We, We) * (1.f / pos_pdf);
  cw[0] = z0;
  uint32_t n = 1;
  V3 prev_f = v3(1.f, 1.f, 1.f);
  float fwd_dir_pdf = dir_pdf;
  float eps = 0.f;
  for(uint32_t b = 0; b <= c.pp.max_depth && n < kBdptVerts; ++b) {
    BVert& prev = cw[n - 1];
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
      cw[n++] = zb;
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
    if(bs.pdf == 0.f) {
      prev.bwd_pdf = 0.f;
      cw[n++] = z;
      break;
    }
    V3 wi = normalize(bs.w);
    float bwd_dir_pdf = bd_bsdf_pdf<G>(m, g.frame, wo, wi, F_ALL);   // camera_f_pdf(wo, wi)
    prev.bwd_pdf = bwd_dir_pdf * fabsf(dot(prev.nn, wo)) / dist2;
    prev_f = bs.f;
    fwd_dir_pdf = bs.pdf;
    o = z.p;
    d = wi;
    eps = g.eps;
    cw[n++] = z;
  }
  return n;
}

// The path of s light and t camera vertices, as path_weight indexes it:
// x[0 .. s-1] = light vertices, x[s .. s+t-1] = camera vertices in reverse.
struct BdptPath {
  const BVert* lw;
  const BVert* cw;
  const BVert* first_light;    // replaces lw[0] (s == 1)
  const BVert* first_camera;   // replaces cw[0] (t == 1)
  uint32_t s, t;
  DG_HD const BVert& light_at(uint32_t i) const { return i == 0 ? *first_light : lw[i]; }
  DG_HD const BVert& camera_at(uint32_t i) const { return i == 0 ? *first_camera : cw[i]; }
  DG_HD const BVert& at(uint32_t i) const {
    return i < s ? light_at(i) : camera_at(t - (i - s + 1));
  }
};

// path_weight (bdpt_renderer.cpp:470-678): the balance heuristic over the
// strategies (s', t') with s' + t' = s + t.
template<bool G>
DG_HD float bdpt_weight(const BdptCtx& c, const DevLight& light, const BdptPath& x) {
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

// One pixel sample (sample_path, bdpt_renderer.cpp:40-94): the camera-side
// value is returned, t = 1 splats go straight to the film.
template<bool G>
DG_HD V3 bdpt_sample(const PtScene& sc, const PtParams& pp, uint32_t pixel, uint32_t sample,
                     float fx, float fy, bool use_t1, float* splat, uint32_t& rays) {
  V3 total = v3(0.f, 0.f, 0.f);
  if(sc.light_count == 0) { return total; }
  BdptCtx c{sc, pp, pixel, sample};
  Rand4 r1 = rand4(pp.seed, pixel, sample, 1);
  uint32_t light_i = distrib_sample(sc.light_cdf, sc.light_count + 1, r1.a);
  float pick = distrib_pdf(sc.light_cdf, sc.light_count + 1, light_i);
  BVert lw[kBdptVerts], cw[kBdptVerts];
  uint32_t ns = pick > 0.f ? bdpt_light_walk<G>(c, light_i, pick, lw, rays) : 0u;
  uint32_t nt = bdpt_camera_walk<G>(c, fx, fy, cw, rays);
  if(ns == 0) { lw[0] = bvert_empty(); }
  if(nt == 0) { return total; }
  // On the device the lanes of a warp run the (s, t) loop in lock step, to
  // the warp's largest walk lengths, so that they take the same connection
  // case together instead of drifting apart by their own walk lengths.
#ifdef __CUDA_ARCH__
  const uint32_t lanes = __activemask();
  const uint32_t s_end = __reduce_max_sync(lanes, ns), t_end = __reduce_max_sync(lanes, nt);
#else
  const uint32_t s_end = ns, t_end = nt;
#endif
  for(uint32_t s = 0; s <= s_end; ++s) {
    for(uint32_t t = 1; t <= t_end; ++t) {
      if(s > ns || t > nt) { continue; }
      if(t == 1 && !use_t1) { continue; }
      if(s + t < pp.min_depth + 2 || s + t > pp.max_depth + 2) { continue; }
      Rand4 rc = rand4(pp.seed, pixel, sample, kBdConnect + 32 * s + t);
      const BVert& last_camera = cw[t - 1];
      uint32_t new_light = light_i;
      // the connection's own end vertices where it makes new ones (s = 1
      // light sample, t = 1 camera point), else the walks' first vertices
      BVert first_light, first_camera;
      const BVert* fl = &lw[0];
      const BVert* fc = &cw[0];
      float sfx = fx, sfy = fy;
      V3 contrib = v3(0.f, 0.f, 0.f);
      if(s > 0 && last_camera.bg != 0) {
        continue;
      } else if(s == 1 && t == 1) {
        if(G && pp.camera == CAMERA_ORTHO) { continue; }   // CAMERA_DIR_BY_POS_DELTA
        float cam_pdf;
        V3 cp = camera_sample_point<G>(pp, rc.a, rc.b, cam_pdf);
        if(cam_pdf == 0.f) { continue; }
        LightSample ls = bd_light_sample<G>(sc, sc.lights[light_i], cp, 0.f, rc.c, rc.d);
        if(ls.pdf == 0.f || is_black(ls.L)) { continue; }
        float We = camera_eval_importance<G>(pp, cp, ls.wi, sfx, sfy);
        if(We == 0.f) { continue; }
        if(pick == 0.f) { continue; }
        ++rays;
        Hit h = bd_trace<true, G>(sc, ls.o, ls.tmin, ls.d, ls.tmax);
        if(h.prim != kMiss) { continue; }
        contrib = ls.L * (We / (cam_pdf * ls.pdf * pick));
      } else if(s == 0 && t >= 2 && last_camera.bg != 0) {
        const DevLight& bl = sc.lights[last_camera.bg - 1u];
        V3 Le = background_radiance(sc, bl, normalize(last_camera.p - cw[t - 2].p));
        if(is_black(Le)) { continue; }
        new_light = last_camera.bg - 1u;
        contrib = Le * last_camera.alpha;
      } else if(s == 0 && t >= 2 && last_camera.light != 0) {
        const DevLight& al = sc.lights[last_camera.light - 1u];
        V3 Le = area_eval_radiance(sc, al, last_camera.p, last_camera.nn, cw[t - 2].p);
        if(is_black(Le)) { continue; }
        new_light = last_camera.light - 1u;
        contrib = Le * last_camera.alpha;
      } else if(s == 0 && t >= 2) {
        continue;
      } else if(s == 1 && t >= 2) {
        uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, rc.a);
        float lp = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
        new_light = li;
        if(lp == 0.f) { continue; }
        const DevLight& l2 = sc.lights[li];
        LightSample ls = bd_light_sample<G>(sc, l2, last_camera.p, last_camera.eps, rc.b, rc.c);
        if(is_black(ls.L) || ls.pdf == 0.f) { continue; }
        ++rays;
        Hit h = bd_trace<true, G>(sc, ls.o, ls.tmin, ls.d, ls.tmax);
        if(h.prim != kMiss) { continue; }
        V3 bwo = normalize(cw[t - 2].p - last_camera.p);
        DevMaterial m = bvert_material(sc, last_camera);
        Frame fr = bvert_frame(last_camera);
        V3 f = bd_bsdf_eval<G>(m, fr, ls.wi, bwo, F_ALL);
        if(is_black(f)) { continue; }
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
      } else if(s >= 2 && t == 1) {
        const BVert& last_light = lw[s - 1];
        CameraPivot cam;
        if(!camera_pivot_importance<G>(pp, last_light.p, rc.a, rc.b, cam) || cam.We == 0.f ||
           cam.pdf == 0.f) {
          continue;
        }
        sfx = cam.fx;
        sfy = cam.fy;
        V3 wi = normalize(lw[s - 2].p - last_light.p);
        V3 wo = normalize(cam.p - last_light.p);
        DevMaterial m = bvert_material(sc, last_light);
        V3 f = bd_bsdf_eval<G>(m, bvert_frame(last_light), wi, wo, F_ALL);
        if(is_black(f)) { continue; }
        ++rays;
        if(!bd_visible<G>(sc, last_light.p, last_light.eps, cam.p, 0.f)) { continue; }
        first_camera = bvert_empty();
        first_camera.p = cam.p;
        first_camera.fwd_pdf = cam.pdf;
        first_camera.alpha = v3(cam.We, cam.We, cam.We);
        fc = &first_camera;
        contrib = last_light.alpha * f *
                  (cam.We * fabsf(dot(last_light.nn, wo)) / (length_sq(cam.p - last_light.p) * cam.pdf));
      } else {
        // s >= 2 && t >= 2
        const BVert& last_light = lw[s - 1];
        ++rays;
        if(!bd_visible<G>(sc, last_light.p, last_light.eps, last_camera.p, last_camera.eps)) {
          continue;
        }
        V3 lwi = normalize(lw[s - 2].p - last_light.p);
        V3 cwo = normalize(cw[t - 2].p - last_camera.p);
        V3 wo = normalize(last_camera.p - last_light.p);
        DevMaterial ml = bvert_material(sc, last_light);
        V3 fl = bd_bsdf_eval<G>(ml, bvert_frame(last_light), lwi, wo, F_ALL);
        if(is_black(fl)) { continue; }
        DevMaterial mc = bvert_material(sc, last_camera);
        V3 fc = bd_bsdf_eval<G>(mc, bvert_frame(last_camera), -wo, cwo, F_ALL);
        if(is_black(fc)) { continue; }
        float geom = fabsf(dot(wo, last_light.nn)) * fabsf(dot(wo, last_camera.nn)) /
                     length_sq(last_light.p - last_camera.p);
        contrib = last_light.alpha * last_camera.alpha * fl * fc * geom;
      }
      if(is_black(contrib)) { continue; }
      BdptPath path{lw, cw, fl, fc, s, t};
      float w = bdpt_weight<G>(c, sc.lights[new_light], path);
      V3 wc = contrib * w;
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
