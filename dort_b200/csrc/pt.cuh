// One path sample of the reference's "pt" renderer, for the device (and, for
// checking without a GPU, the host).
//
// Restates PathRenderer::sample / sample_direct_lighting / estimate_direct*
// (src/dort/path_renderer.cpp:23-206) over the flat device scene:
//   - BSDF: Bsdf (bsdf.cpp:50-242) specialised to the single BxDF that every
//     material in scope adds -- LambertBrdf (lambert_material.cpp:5-35),
//     MirrorBrdf (mirror_material.cpp:5-29), DielectricBxdf
//     (dielectric_material.cpp:32-116, fresnel.cpp:5-47), PhongBrdf
//     (phong_material.cpp:6-106), OrenNayarBrdf (oren_nayar_material.cpp:5-72)
//     and a GGX conductor built on the reference's GGX distribution
//     (microfacet.cpp:19-86; the conductor itself has no reference
//     counterpart);
//   - geometry: the triangle BVH (trace.cuh) plus analytic shapes
//     (shapes.cuh);
//   - lights: DiffuseLight on a triangle, sphere or disk (diffuse_light.cpp:40-111,
//     shape.cpp:4-26, triangle.cpp:62-80, sphere_shape.cpp:74-121),
//     PointLight (point_light.cpp:19-31), DirectionalLight
//     (directional_light.cpp:28-42), InfiniteLight (infinite_light.cpp:5-65),
//     EnvironmentLight (environment_light.cpp);
//   - cameras: PinholeCamera, OrthoCamera and ThinLensCamera
//     ::sample_ray_importance (pinhole_camera.cpp:13-31, ortho_camera.cpp:13-26,
//     thin_lens_camera.cpp:15-33);
//   - light choice: DiscreteDistrib1d over approximate powers
//     (discrete_distrib_1d.cpp, scene.cpp:20-28).
// Random numbers come from Philox keyed by (seed, pixel, sample, block); see
// philox.cuh for the dimension layout.
//
// Template flag G ("general"): the functions that depend on scene features
// are instantiated twice.  G = false compiles only what a triangle scene with
// triangle and sky lights, a pinhole camera and the materials Lambert,
// mirror, dielectric (outside ior 1, not thin), Phong and conductor needs;
// G = true adds analytic shapes, point and directional lights, orthographic
// and thin-lens cameras, Oren-Nayar and the general dielectric.  The host
// picks the instantiation per scene and camera (scene_needs_general), so the
// common case does not pay in registers for code it never runs.
#pragma once
#include <cmath>

#include "philox.cuh"
#include "pt_scene.h"
#include "trace.cuh"
#include "pt_math.cuh"
#include "shapes.cuh"

namespace dort_gpu {

// ---- BSDF -------------------------------------------------------------------

// Shading frame of a triangle hit (bsdf.cpp:50-66 with the DiffGeom of
// TriangleUv::hit, triangle.cpp:137-171, default uvs: dpdu = e1).
struct Frame {
  V3 n, s, t;
  DG_HD V3 to_local(V3 v) const { return v3(dot(s, v), dot(t, v), dot(n, v)); }
  DG_HD V3 to_world(V3 v) const { return s * v.x + t * v.y + n * v.z; }
};

DG_HD bool bxdf_matches(uint32_t flags, uint32_t request) {
  return (flags & (request & F_MODES)) && (flags & (request & F_LOBES));
}

struct BsdfSample {
  V3 f;
  V3 w;        // world direction
  float pdf;
  uint32_t flags;
};

// GGX distribution (microfacet.cpp:19-36, 38-58, 60-86 -- the reference's
// sample_m always takes the GGX branch).
DG_HD float ggx_d(V3 m, float alpha) {
  float c2 = m.z * m.z;
  float s2 = 1.f - c2;
  float t2 = s2 / c2;
  return kInvPi * sq(alpha) / sq(c2 * (sq(alpha) + t2));
}
DG_HD float ggx_g1(V3 v, V3 m, float alpha) {
  if(dot(v, m) * v.z <= 0.f) { return 0.f; }
  float c2 = v.z * v.z;
  float t2 = (1.f - c2) / c2;
  return 2.f / (1.f + sqrtf(1.f + sq(alpha) * t2));
}
DG_HD V3 ggx_sample_m(float u1, float u2, float alpha, float& pdf) {
  float ct = 1.f / sqrtf((sq(alpha) * u1) / (1.f - u1) + 1.f);
  float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  float sp, cp;
  DG_SINCOSPI(2.f * u2, sp, cp);
  V3 m = v3(st * sp, st * cp, ct);
  pdf = ggx_d(m, alpha) * ct;
  return m;
}
DG_HD V3 schlick(V3 f0, float cos_i) {
  float x = 1.f - fminf(fabsf(cos_i), 1.f);
  float x2 = x * x;
  float k = x2 * x2 * x;
  return v3(f0.x + (1.f - f0.x) * k, f0.y + (1.f - f0.y) * k, f0.z + (1.f - f0.z) * k);
}

// Conductor (no reference counterpart): f = F(wi.m) D(m) G1(wi) G1(wo) /
// (4 |cos wi| |cos wo|), m sampled from D(m) cos(m) mirrored into the
// hemisphere of wo, pdf = D(m) |cos m| / (4 |wo.m|).
DG_HD V3 conductor_f(const DevMaterial& m, V3 wi, V3 wo) {
  if(wi.z * wo.z <= 0.f) { return v3(0.f, 0.f, 0.f); }
  V3 h = wi + wo;
  if(is_black(h)) { return v3(0.f, 0.f, 0.f); }
  h = normalize(h);
  if(h.z < 0.f) { h = -h; }
  float a = m.p0;
  float d = ggx_d(h, a);
  float g = ggx_g1(wi, h, a) * ggx_g1(wo, h, a);
  V3 F = schlick(v3p(m.c), dot(wi, h));
  return F * (d * g / (4.f * fabsf(wi.z) * fabsf(wo.z)));
}
DG_HD float conductor_pdf(const DevMaterial& m, V3 wi, V3 wo) {
  if(wi.z * wo.z <= 0.f) { return 0.f; }
  V3 h = wi + wo;
  if(is_black(h)) { return 0.f; }
  h = normalize(h);
  if(h.z < 0.f) { h = -h; }
  float dwo = fabsf(dot(wo, h));
  if(dwo == 0.f) { return 0.f; }
  return ggx_d(h, m.p0) * fabsf(h.z) / (4.f * dwo);
}

// OrenNayarBrdf::eval_f (oren_nayar_material.cpp:5-38); m.p0 = sigma^2 terms
// A and B precomputed as p1, p2.
DG_HD V3 oren_nayar_f(const DevMaterial& m, V3 wi, V3 wo) {
  float ci = fabsf(wi.z), co = fabsf(wo.z);
  if(ci == 0.f || co == 0.f) { return v3(0.f, 0.f, 0.f); }
  float a = m.p1, b = m.p2;
  if(ci >= 0.99f || co >= 0.99f) { return v3p(m.c) * (kInvPi * a); }
  // Bsdf::sin_theta / sin_phi / cos_phi (bsdf.hpp:220-247)
  float si = sqrtf(fmaxf(0.f, 1.f - wi.z * wi.z));
  float so = sqrtf(fmaxf(0.f, 1.f - wo.z * wo.z));
  float spi = wi.y / si, cpi = wi.x / si, spo = wo.y / so, cpo = wo.x / so;
  float cos_dphi = cpi * cpo + spi * spo;
  float sin_alpha, tan_beta;
  if(ci >= co) {
    sin_alpha = so;
    tan_beta = si / ci;
  } else {
    sin_alpha = si;
    tan_beta = so / co;
  }
  return v3p(m.c) * (kInvPi * (a + b * fmaxf(0.f, cos_dphi) * sin_alpha * tan_beta));
}

// Bxdf::eval_f for the resolved BxDF of `m` (local directions).
template<bool G>
DG_HD V3 bxdf_eval(const DevMaterial& m, V3 wi, V3 wo, uint32_t request) {
  switch(m.kind) {
    case DORT_MAT_LAMBERT:
      return v3p(m.c) * kInvPi;
    case DORT_MAT_PHONG: {
      // phong_material.cpp:22-38
      bool s_diff = m.p1 < 1.f && (request & F_DIFF);
      bool s_glossy = m.p1 > 0.f && (request & F_GLOSSY);
      V3 diffuse = v3p(m.c) * kInvPi;
      if(!s_glossy) { return diffuse; }
      V3 wo_r = v3(-wo.x, -wo.y, wo.z);
      float ca = dot(wo_r, wi);
      V3 glossy = ca < 0.f ? v3(0.f, 0.f, 0.f)
          : v3p(m.c2) * ((m.p0 + 2.f) * kInvTwoPi * powf(ca, m.p0));
      return s_diff ? diffuse + glossy : glossy;
    }
    case DORT_MAT_CONDUCTOR:
      return conductor_f(m, wi, wo);
    case DORT_MAT_OREN_NAYAR:
      return G ? oren_nayar_f(m, wi, wo) : v3(0.f, 0.f, 0.f);
    default:
      return v3(0.f, 0.f, 0.f);   // mirror, dielectric: delta only
  }
}

// Bxdf light_f_pdf / symmetric_f_pdf (local directions).
template<bool G>
DG_HD float bxdf_pdf(const DevMaterial& m, V3 wg, V3 wf, uint32_t request) {
  switch(m.kind) {
    case DORT_MAT_LAMBERT:
      return cosine_hemisphere_pdf(wg.z);
    case DORT_MAT_PHONG: {
      // phong_material.cpp:80-96 (lerp(t, a, b) = (1 - t) a + t b)
      V3 wr = v3(-wf.x, -wf.y, wf.z);
      float ca = fabsf(dot(wr, wg));
      float dp = cosine_hemisphere_pdf(wg.z);
      float gp = power_cosine_hemisphere_pdf(ca, m.p0);
      if((request & F_GLOSSY) && (request & F_DIFF)) {
        return (1.f - m.p1) * gp + m.p1 * dp;
      } else if(request & F_GLOSSY) {
        return gp;
      } else if(request & F_DIFF) {
        return dp;
      }
      return 0.f;
    }
    case DORT_MAT_CONDUCTOR:
      return conductor_pdf(m, wg, wf);
    case DORT_MAT_OREN_NAYAR:
      return G ? cosine_hemisphere_pdf(wg.z) : 0.f;
    default:
      return 0.f;
  }
}

// fresnel.cpp:5-32
DG_HD bool refract_dielectric(V3 w, V3& wt, float ior_refl, float ior_trans) {
  float eta = ior_refl / ior_trans;
  float xt = w.x * eta, yt = w.y * eta;
  float st2 = xt * xt + yt * yt;
  if(st2 >= 1.f) { return false; }
  float zt = sqrtf(1.f - st2);
  wt = v3(-xt, -yt, -copysignf(zt, w.z));
  return true;
}
DG_HD float fresnel_dielectric(float cr, float ct, float ir, float it) {
  float tr = it * cr, rt = ir * ct, rr = ir * cr, tt = it * ct;
  float rpa = (tr - rt) / (tr + rt);
  float rpe = (rr - tt) / (rr + tt);
  return 0.5f * (rpa * rpa + rpe * rpe);
}

// Bxdf::sample_light_f (local w_fix = wo); returns f, fills w (local), pdf,
// flags.  Sampling as the reference's per-BxDF code.
template<bool G>
DG_HD V3 bxdf_sample(const DevMaterial& m, V3 wf, uint32_t request, float u, float v,
                     float uc, V3& wg, float& pdf, uint32_t& flags) {
  V3 zero = v3(0.f, 0.f, 0.f);
  switch(m.kind) {
    case DORT_MAT_LAMBERT: {
      wg = cosine_hemisphere_sample(u, v);
      pdf = cosine_hemisphere_pdf(wg.z);
      flags = F_REFL | F_DIFF;
      wg.z = copysignf(wg.z, wf.z);
      return v3p(m.c) * kInvPi;
    }
    case DORT_MAT_MIRROR: {
      wg = v3(-wf.x, -wf.y, wf.z);
      pdf = 1.f;
      flags = F_DELTA | F_REFL;
      if(wf.z == 0.f) { return zero; }
      return v3p(m.c) * (1.f / fabsf(wf.z));
    }
    case DORT_MAT_OREN_NAYAR: {
      // OrenNayarBrdf::sample_symmetric_f (oren_nayar_material.cpp:40-50)
      if(!G) { flags = 0; pdf = 0.f; return zero; }
      wg = cosine_hemisphere_sample(u, v);
      pdf = cosine_hemisphere_pdf(wg.z);
      wg.z = copysignf(wg.z, wf.z);
      flags = F_REFL | F_DIFF;
      return oren_nayar_f(m, wf, wg);
    }
    case DORT_MAT_DIELECTRIC: {
      // dielectric_material.cpp:33-99 with fix_is_light = false; m.p0 =
      // ior_inside, m.p1 = ior_outside, m.p2 != 0: thin slab; get_iors (:101-111)
      bool s_refl = request & F_REFL, s_trans = request & F_TRANS;
      bool thin = G && m.p2 != 0.f;
      float ior_out = G ? m.p1 : 1.f;
      float ir, it;
      if(thin || wf.z >= 0.f) { ir = ior_out; it = m.p0; } else { ir = m.p0; it = ior_out; }
      float cr = fabsf(wf.z);
      V3 w_reflect = v3(-wf.x, -wf.y, wf.z);
      V3 w_trans;
      if(!refract_dielectric(wf, w_trans, ir, it)) {
        if(!s_refl) { flags = 0; pdf = 0.f; return zero; }
        flags = F_DELTA | F_REFL;
        pdf = 1.f;
        wg = w_reflect;
        return v3p(m.c) * (1.f / cr);
      }
      float ct = fabsf(w_trans.z);
      float fr = fresnel_dielectric(cr, ct, ir, it);
      float r = thin ? 1.f - sq(1.f - fr) / (1.f - sq(fr)) : fr;
      float t = 1.f - r;
      bool reflect = uc <= r && s_refl;
      bool transmit = uc > r && s_trans;
      float rp = s_trans ? r : 1.f;
      float tp = s_refl ? t : 1.f;
      if(reflect) {
        flags = F_DELTA | F_REFL;
        pdf = rp;
        wg = w_reflect;
        return v3p(m.c) * (r / cr);
      } else if(transmit && thin) {
        flags = F_DELTA | F_TRANS;
        pdf = tp;
        wg = -wf;
        return v3p(m.c2) * (t / cr);
      } else if(transmit) {
        flags = F_DELTA | F_TRANS;
        pdf = tp;
        wg = w_trans;
        return v3p(m.c2) * (t / ct);
      }
      flags = 0;
      pdf = 0.f;
      return zero;
    }
    case DORT_MAT_PHONG: {
      // phong_material.cpp:40-78
      bool glossy;
      if((request & F_DIFF) && (request & F_GLOSSY)) {
        glossy = uc < m.p1;
      } else {
        glossy = request & F_GLOSSY;
      }
      if(glossy) {
        V3 rw = v3(-wf.x, -wf.y, wf.z);
        V3 rs, rt;
        coordinate_system(rw, rs, rt);
        V3 rel = power_cosine_hemisphere_sample(u, v, m.p0);
        wg = rw * rel.z + rs * rel.x + rt * rel.y;
        flags = F_REFL | F_GLOSSY;
      } else {
        wg = cosine_hemisphere_sample(u, v);
        flags = F_REFL | F_DIFF;
      }
      wg.z = copysignf(wg.z, wf.z);
      pdf = bxdf_pdf<G>(m, wg, wf, request);
      return bxdf_eval<G>(m, wg, wf, request);
    }
    case DORT_MAT_CONDUCTOR: {
      float pm;
      V3 h = ggx_sample_m(u, v, m.p0, pm);
      if(wf.z < 0.f) { h.z = -h.z; }
      float d = dot(wf, h);
      wg = 2.f * d * h - wf;
      flags = F_REFL | F_GLOSSY;
      if(wg.z * wf.z <= 0.f || d == 0.f) { pdf = 0.f; return zero; }
      pdf = pm / (4.f * fabsf(d));
      return conductor_f(m, wg, wf);
    }
    default:
      flags = 0;
      pdf = 0.f;
      return zero;
  }
}

// Bsdf::sample_light_f (bsdf.cpp:95-192) for a one-BxDF Bsdf.
template<bool G>
DG_HD BsdfSample bsdf_sample(const DevMaterial& m, const Frame& fr, V3 wo, uint32_t request,
                             float u, float v, float uc) {
  BsdfSample s;
  s.f = v3(0.f, 0.f, 0.f);
  s.w = v3(0.f, 0.f, 0.f);
  s.pdf = 0.f;
  s.flags = 0;
  if(!bxdf_matches(m.bxdf_flags, request)) { return s; }
  V3 wf = fr.to_local(wo);
  V3 wg;
  float pdf = 0.f;
  uint32_t flags = 0;
  V3 f = bxdf_sample<G>(m, wf, request, u, v, uc, wg, pdf, flags);
  if(pdf == 0.f) { return s; }
  s.flags = flags;
  s.w = fr.to_world(wg);
  s.pdf = pdf;
  // shading_to_geom: shading and geometric normals coincide (no vertex normals)
  float dn = fabsf(dot(fr.n, s.w));
  s.f = (dn * dn == 0.f) ? v3(0.f, 0.f, 0.f) : f;
  return s;
}

// Bsdf::eval_f (bsdf.cpp:72-93).
template<bool G>
DG_HD V3 bsdf_eval(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo, uint32_t request) {
  V3 wi_l = fr.to_local(wi), wo_l = fr.to_local(wo);
  bool reflection = wo_l.z * wi_l.z > 0.f;
  uint32_t er = request & ((F_LOBES & ~F_DELTA) | (reflection ? F_REFL : F_TRANS));
  if(!(er & F_MODES)) { return v3(0.f, 0.f, 0.f); }
  if(!bxdf_matches(m.bxdf_flags, er)) { return v3(0.f, 0.f, 0.f); }
  V3 f = bxdf_eval<G>(m, wi_l, wo_l, er);
  float dn = fabsf(dot(fr.n, wi));
  return (dn * dn == 0.f) ? v3(0.f, 0.f, 0.f) : f;
}

// Bsdf::light_f_pdf (bsdf.cpp:194-225).
template<bool G>
DG_HD float bsdf_pdf(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo, uint32_t request) {
  if(!bxdf_matches(m.bxdf_flags, request)) { return 0.f; }
  return bxdf_pdf<G>(m, fr.to_local(wi), fr.to_local(wo), request);
}

// ---- scene access ---------------------------------------------------------------

// The analytic shapes (a short list, each tested in its own space against the
// closest t so far).
template<bool ANY_HIT>
DG_HD Hit trace_shapes(const PtScene& sc, V3 o, float t_min, V3 d,
                                                  float t_max, Hit h) {
  float best = h.prim == kMiss ? t_max : h.t;
  for(uint32_t k = 0; k < sc.shape_count; ++k) {
    const DevShape& s = sc.shapes[k];
    V3 ol = xf_point(s.inv, o), dl = xf_vec(s.inv, d);
    float t;
    uint32_t face;
    if(shape_hit<ANY_HIT>(s, ol, dl, t_min, best, t, face)) {
      h.t = t;
      h.b1 = float(face);
      h.b2 = 0.f;
      h.prim = sc.shape_base + k;
      if(ANY_HIT) { return h; }
      best = t;
    }
  }
  return h;
}

// Scene::intersect / intersect_p (scene.cpp:8-18) over the flat scene: the
// triangle BVH, then the analytic shapes.  A shape hit has prim = shape_base +
// its index and b1 = the cube face.
template<bool ANY_HIT, bool G>
DG_HD Hit scene_trace(const PtScene& sc, V3 o, float t_min, V3 d, float t_max) {
  // the general instantiation also serves scenes built watertight
  Hit h = trace_ray<ANY_HIT, false, G ? kTriByScene : kTriMt>(sc.trace, o.x, o.y, o.z, t_min,
                                                             d.x, d.y, d.z, t_max);
  if(!G || sc.shape_count == 0 || (ANY_HIT && h.prim != kMiss)) { return h; }
  return trace_shapes<ANY_HIT>(sc, o, t_min, d, t_max, h);
}

// Material index of a hit primitive.
template<bool G>
DG_HD uint32_t prim_material(const PtScene& sc, uint32_t prim) {
  if(G && prim >= sc.shape_base) { return sc.shapes[prim - sc.shape_base].mat; }
  return DG_AS_UINT(DG_LDG(&sc.shade[3 * size_t(prim)].w));
}

struct SurfaceHit {
  V3 p, n;          // point, unit geometric normal (triangles: cross(e2, e1))
  Frame frame;
  float eps;        // ray epsilon (triangles |1e-3 t|)
  uint32_t tri;     // hit prim (a shape's is >= shape_base)
  uint32_t mat;
  uint32_t light;   // light index + 1, 0 if not emissive
};

// DiffGeom of an analytic shape hit (the shape's hit, transformed by
// Transform::apply(DiffGeom), transform.cpp:15-25).  The BSDF frame is any
// frame around the normal: every BxDF here is isotropic.
DG_HD SurfaceHit shape_surface(const PtScene& sc, const Hit& h, V3 o, V3 d) {
  SurfaceHit s;
  const DevShape& sh = sc.shapes[h.prim - sc.shape_base];
  V3 ol = xf_point(sh.inv, o), dl = xf_vec(sh.inv, d);
  V3 pl = madd_rn(ol, dl, h.t);
  V3 nl = shape_local_normal(sh, pl, uint32_t(h.b1));
  s.p = xf_point(sh.m, pl);
  s.n = normalize(xf_normal(sh.inv, nl));
  s.eps = shape_ray_epsilon(sh, h.t);
  s.tri = h.prim;
  s.mat = sh.mat;
  s.light = sh.light;
  s.frame.n = s.n;
  coordinate_system(s.n, s.frame.s, s.frame.t);
  return s;
}

// Surface at the closest hit h of the ray (o, d).
template<bool G>
DG_HD SurfaceHit surface_at(const PtScene& sc, const Hit& h, V3 o, V3 d) {
  if(G && h.prim >= sc.shape_base) { return shape_surface(sc, h, o, d); }
  SurfaceHit s;
  const float4* sh = sc.shade + 3 * size_t(h.prim);
  float4 a = DG_LDG(sh), b = DG_LDG(sh + 1), c = DG_LDG(sh + 2);
  V3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
  V3 e1 = p1 - p0, e2 = p2 - p0;
  float b0 = 1.f - h.b1 - h.b2;
  s.p = b0 * p0 + h.b1 * p1 + h.b2 * p2;
  s.n = normalize(cross(e2, e1));
  s.eps = fabsf(1e-3f * h.t);
  s.tri = h.prim;
  s.mat = DG_AS_UINT(a.w);
  s.light = DG_AS_UINT(b.w);
  s.frame.n = s.n;
  float len = length(e1);
  if(len < 1e-9f) {
    coordinate_system(s.n, s.frame.s, s.frame.t);
  } else {
    s.frame.s = e1 * (1.f / len);
    s.frame.t = cross(s.n, s.frame.s);
  }
  return s;
}

// Material of a hit, with the optional per-triangle albedo override.
DG_HD DevMaterial material_at(const PtScene& sc, const SurfaceHit& s) {
  DevMaterial m = sc.mats[s.mat];
  if(sc.tri_albedo && m.bxdf_flags && s.tri < sc.shape_base) {
    const float* a = sc.tri_albedo + 3 * size_t(s.tri);
    m.c[0] = a[0]; m.c[1] = a[1]; m.c[2] = a[2];
    if(m.kind == DORT_MAT_LAMBERT && a[0] == 0.f && a[1] == 0.f && a[2] == 0.f) {
      m.bxdf_flags = 0;
    }
  }
  return m;
}

DG_HD V3 light_radiance(const PtScene& sc, const DevLight& l) {
  if(sc.tri_emission && l.kind == LIGHT_TRI) {
    return v3p(sc.tri_emission + 3 * size_t(l.tri));
  }
  return v3p(l.L);
}

// DiffuseLight::eval_radiance (diffuse_light.cpp:85-94)
DG_HD V3 area_eval_radiance(const PtScene& sc, const DevLight& l, V3 p, V3 n, V3 pivot) {
  return dot(n, pivot - p) >= 0.f ? light_radiance(sc, l) : v3(0.f, 0.f, 0.f);
}

// DiscreteDistrib1d::sample / pdf (discrete_distrib_1d.cpp:22-41)
DG_HD uint32_t distrib_sample(const float* cdf, uint32_t n_plus_1, float u) {
  uint32_t begin = 0, end = n_plus_1 - 1;
  while(begin + 1 < end) {
    uint32_t mid = begin + (end - begin) / 2;
    if(cdf[mid] < u) { begin = mid; } else { end = mid; }
  }
  return begin;
}
DG_HD float distrib_pdf(const float* cdf, uint32_t n_plus_1, uint32_t i) {
  if(i + 1 >= n_plus_1) { return 0.f; }
  return cdf[i + 1] - cdf[i];
}

// EnvironmentLight helpers (environment_light.cpp:104-158)
DG_HD V3 env_dir_from_uv(const DevEnv& e, float du, float dv, float& sin_t) {
  // theta = pi dv, phi = 2 pi (du - 1/2)
  float ct, st, cp, sp;
  DG_SINCOSPI(dv, st, ct);
  DG_SINCOSPI(2.f * du - 1.f, sp, cp);
  sin_t = clampf(st, 0.f, 1.f);
  return v3p(e.up) * ct + v3p(e.s) * (st * cp) + v3p(e.t) * (st * sp);
}
DG_HD void env_uv_from_dir(const DevEnv& e, V3 d, float& du, float& dv, float& sin_t) {
  float up = dot(d, v3p(e.up)), s = dot(d, v3p(e.s)), t = dot(d, v3p(e.t));
  float phi = atan2f(t, s);
  float theta = acosf(clampf(up, -1.f, 1.f));
  sin_t = sqrtf(fmaxf(0.f, 1.f - up * up));
  du = phi * kInvTwoPi + 0.5f;
  dv = theta * kInvPi;
}
DG_HD V3 env_radiance_uv(const DevEnv& e, float du, float dv) {
  float fx = floorf(du * float(e.w)), fy = floorf(dv * float(e.h));
  if(!(fx >= 0.f) || !(fy >= 0.f)) { return v3(0.f, 0.f, 0.f); }
  if(fx >= float(e.w) || fy >= float(e.h)) { return v3(0.f, 0.f, 0.f); }
  const float* p = e.rgb + 3 * (size_t(fy) * e.w + size_t(fx));
  return v3(e.scale[0] * DG_LDG(p), e.scale[1] * DG_LDG(p + 1), e.scale[2] * DG_LDG(p + 2));
}
DG_HD float env_dir_uv_pdf(const DevEnv& e, float du, float dv) {
  float x = du * float(e.w), y = dv * float(e.h);
  float fx = floorf(x), fy = floorf(y);
  if(!(fx >= 0.f) || !(fy >= 0.f) || fx >= float(e.w) || fy >= float(e.h)) { return 0.f; }
  return DG_LDG(e.pdfs + size_t(fy) * e.w + size_t(fx)) * float(e.w * e.h);
}
DG_HD float env_dir_pdf(const DevEnv& e, V3 d) {
  float du, dv, st;
  env_uv_from_dir(e, d, du, dv, st);
  if(st == 0.f) { return 0.f; }
  return env_dir_uv_pdf(e, du, dv) / (2.f * kPi * kPi * st);
}
// One draw from an alias table of n entries (scene_build.cpp build_alias):
// u picks an entry and its fraction decides between the entry and its alias;
// the fraction, rescaled, is returned in `rest` as a fresh uniform (about 14
// bits for tables of 1024 entries: the position inside a texel).
DG_HD uint32_t alias_draw(const float2* t, uint32_t n, float u, float& rest) {
  float x = u * float(n);
  uint32_t i = x < float(n) ? uint32_t(x) : n - 1u;
  float f = x - float(i);
  float2 a = DG_LDG(t + i);
  if(f < a.x) {
    rest = f / a.x;
    return i;
  }
  rest = (f - a.x) / (1.f - a.x);
  return DG_AS_UINT(a.y);
}

// A direction of the environment light drawn from its texel distribution:
// the row by its alias table, the column by the row's, the point inside the
// texel uniform (the distribution PiecewiseDistrib2d::sample draws by
// inverting its CDFs, piecewise_distrib_2d.cpp:37-70, in two table reads
// instead of two binary searches).
DG_HD V3 env_sample_dir(const DevEnv& e, float u, float v, float& du, float& dv, float& pdf) {
  float rx, ry;
  uint32_t yi = alias_draw(e.row_alias, e.h, v, ry);
  uint32_t xi = alias_draw(e.col_alias + size_t(e.w) * yi, e.w, u, rx);
  const float below_one = 0.99999994f;
  du = (float(xi) + fminf(rx, below_one)) / float(e.w);
  dv = (float(yi) + fminf(ry, below_one)) / float(e.h);
  float st;
  V3 d = env_dir_from_uv(e, du, dv, st);
  pdf = st == 0.f ? 0.f : env_dir_uv_pdf(e, du, dv) / (2.f * kPi * kPi * st);
  return d;
}

DG_HD V3 background_radiance(const PtScene& sc, const DevLight& l, V3 dir) {
  if(l.kind == LIGHT_INFINITE) { return v3p(l.L); }
  float du, dv, st;
  env_uv_from_dir(sc.env, dir, du, dv, st);
  return env_radiance_uv(sc.env, du, dv);
}

// DiffuseLight::pivot_radiance_pdf (diffuse_light.cpp:104-110) on an analytic
// shape, in shape space.
DG_HD float shape_light_pivot_pdf(const PtScene& sc, const DevLight& l, V3 wi, V3 pivot) {
  const DevShape& sh = sc.light_shapes[l.tri];
  return shape_pivot_pdf(sh, xf_point(sh.inv, pivot), normalize(xf_vec(sh.inv, wi)));
}

DG_HD bool light_is_area(const DevLight& l) { return l.kind == LIGHT_TRI || l.kind == LIGHT_SHAPE; }
DG_HD bool light_is_background(const DevLight& l) {
  return l.kind == LIGHT_INFINITE || l.kind == LIGHT_ENV;
}

// Light::pivot_radiance_pdf
template<bool G>
DG_HD float light_pivot_pdf(const PtScene& sc, const DevLight& l, V3 wi, V3 pivot) {
  if(l.kind == LIGHT_INFINITE) { return kInvFourPi; }
  if(l.kind == LIGHT_ENV) { return env_dir_pdf(sc.env, wi); }
  if(G) {
    if(l.kind == LIGHT_POINT) { return length_sq(v3p(l.p0) - pivot); }  // point_light.cpp:50-52
    if(l.kind == LIGHT_DIR) { return 1.f; }                             // directional_light.cpp:60-62
    if(l.kind == LIGHT_SHAPE) { return shape_light_pivot_pdf(sc, l, wi, pivot); }
  }
  // Shape::point_pivot_pdf (shape.cpp:15-26) on the light's triangle
  V3 w = normalize(wi);
  float4 a = make_float4(l.p0[0], l.p0[1], l.p0[2], 0.f);
  float4 e1 = make_float4(l.e1[0], l.e1[1], l.e1[2], 0.f);
  float4 e2 = make_float4(l.e2[0], l.e2[1], l.e2[2], 0.f);
  float t, b1, b2;
  if(!mt_exact(a, e1, e2, pivot.x, pivot.y, pivot.z, w.x, w.y, w.z, 0.f, INFINITY, t, b1, b2)) {
    return 0.f;
  }
  V3 pt = pivot + w * t;
  return (1.f / l.area) * length_sq(pt - pivot) / fabsf(dot(w, v3p(l.nn)));
}

struct LightSample {
  V3 L, wi;
  float pdf;
  // shadow segment
  V3 o, d;
  float tmin, tmax;
  // the sampled light point, its normal and ray epsilon (area and point
  // lights; bidirectional connections)
  V3 p, nn;
  float p_eps;
};

// DiffuseLight::sample_pivot_radiance (diffuse_light.cpp:40-68) on an
// analytic shape: sampled in shape space, emitting to the side of the shape's
// normal.
DG_HD LightSample shape_light_sample(const PtScene& sc, const DevLight& l, V3 pivot,
                                     float pivot_eps, float u, float v) {
  LightSample s;
  const DevShape& sh = sc.light_shapes[l.tri];
  V3 pl = xf_point(sh.inv, pivot);
  V3 n;
  float eps;
  V3 ptl = shape_sample_pivot(sh, pl, u, v, n, s.pdf, eps);
  V3 swi = normalize(ptl - pl);
  V3 pt = xf_point(sh.m, ptl);
  float dist = length(pt - pivot);
  s.wi = normalize(pt - pivot);
  s.o = pivot;
  s.d = (pt - pivot) * (1.f / dist);
  s.tmin = pivot_eps;
  s.tmax = dist - eps;
  s.L = dot(swi, n) < 0.f ? light_radiance(sc, l) : v3(0.f, 0.f, 0.f);
  s.p = pt;
  s.nn = normalize(xf_normal(sh.inv, n));
  s.p_eps = eps;
  return s;
}

// Light::sample_pivot_radiance for every light kind.
template<bool G>
DG_HD LightSample light_sample(const PtScene& sc, const DevLight& l, V3 pivot, float pivot_eps,
                               float u, float v) {
  LightSample s;
  s.L = v3(0.f, 0.f, 0.f);
  s.pdf = 0.f;
  if(l.kind == LIGHT_TRI) {
    // Triangle::sample_point (triangle.cpp:62-76), Shape::sample_point_pivot
    float sr = sqrtf(u);
    float b1 = 1.f - sr, b2 = v * sr;
    V3 pt = v3p(l.p0) + b1 * v3p(l.e1) + b2 * v3p(l.e2);
    V3 n = v3p(l.nn);
    V3 to = pivot - pt;
    s.pdf = (1.f / l.area) * length_sq(to) / fabsf(dot(n, normalize(to)));
    V3 wi = normalize(pt - pivot);
    s.wi = wi;
    // ShadowTest::init_point_point (light.cpp:40-49)
    float dist = length(pt - pivot);
    s.o = pivot;
    s.d = (pt - pivot) * (1.f / dist);
    s.tmin = pivot_eps;
    s.tmax = dist - 1e-3f;
    s.L = dot(wi, n) < 0.f ? light_radiance(sc, l) : v3(0.f, 0.f, 0.f);
    s.p = pt;
    s.nn = n;
    s.p_eps = 1e-3f;
  } else if(G && l.kind == LIGHT_SHAPE) {
    s = shape_light_sample(sc, l, pivot, pivot_eps, u, v);
  } else if(G && l.kind == LIGHT_POINT) {
    // PointLight::sample_pivot_radiance (point_light.cpp:19-31)
    V3 pt = v3p(l.p0);
    float dist = length(pt - pivot);
    s.wi = normalize(pt - pivot);
    s.pdf = length_sq(pt - pivot);
    s.o = pivot;
    s.d = (pt - pivot) * (1.f / dist);
    s.tmin = pivot_eps;
    s.tmax = dist;
    s.L = v3p(l.L);
    s.p = pt;
    s.nn = -s.wi;     // point_light.cpp:27
    s.p_eps = 0.f;
  } else if(G && l.kind == LIGHT_DIR) {
    // DirectionalLight::sample_pivot_radiance (directional_light.cpp:28-42)
    s.wi = -v3p(l.nn);
    s.pdf = 1.f;
    s.o = pivot;
    s.d = normalize(s.wi);
    s.tmin = pivot_eps;
    s.tmax = INFINITY;
    s.L = v3p(l.L);
  } else {
    V3 wi;
    if(l.kind == LIGHT_INFINITE) {
      wi = uniform_sphere_sample(u, v);
      s.pdf = kInvFourPi;
      s.L = v3p(l.L);
    } else {
      float du, dv;
      wi = env_sample_dir(sc.env, u, v, du, dv, s.pdf);
      s.L = env_radiance_uv(sc.env, du, dv);
    }
    s.wi = wi;
    s.o = pivot;
    s.d = normalize(wi);
    s.tmin = pivot_eps;
    s.tmax = INFINITY;
  }
  return s;
}

// ---- the path ---------------------------------------------------------------------

// Observer of the terms a path adds to its sample value, in path order; the
// adjoint replays a path with an observer that attributes derivatives, the
// forward renderers pass this no-op.
//   emission(light tri, throughput, Le)  adds throughput * Le
//   background(c)                        adds c
//   vertex(tri, material)                a scattering vertex starts; every
//                                        later term is linear in its BSDF
//   direct(light tri or kMiss, c)        adds c (a direct-lighting term)
struct NoTape {
  DG_HD void emission(uint32_t, V3, V3) {}
  DG_HD void background(V3) {}
  DG_HD void vertex(uint32_t, const DevMaterial&) {}
  DG_HD void direct(uint32_t, V3) {}
};

struct PathResult {
  V3 L;
  uint32_t rays;   // closest-hit + shadow rays traced
};

// Radiance that area light `li` sends along a BSDF-strategy ray from p whose
// closest hit is h: only a hit on the light's own primitive counts
// (estimate_direct_from_bsdf, path_renderer.cpp:158-166).
template<bool G>
DG_HD V3 area_light_hit_radiance(const PtScene& sc, uint32_t li, const Hit& h, V3 p, V3 wi) {
  if(h.prim == kMiss) { return v3(0.f, 0.f, 0.f); }
  SurfaceHit g = surface_at<G>(sc, h, p, wi);
  if(g.light != li + 1) { return v3(0.f, 0.f, 0.f); }
  return area_eval_radiance(sc, sc.lights[li], g.p, g.n, p);
}

// Camera ray of film position (fx, fy) for sample `sample` of `pixel`; the
// thin lens draws its lens point from the camera block of the sample.
template<bool G>
DG_HD void camera_ray(const PtParams& pp, uint32_t pixel, uint32_t sample, float fx, float fy,
                      V3& o, V3& d) {
  float w = float(pp.width), h = float(pp.height);
  if(G && pp.camera == CAMERA_ORTHO) {
    // OrthoCamera::sample_ray_importance / get_plane_pos (ortho_camera.cpp:13-26,84-88)
    float k = pp.ortho_dim / fmaxf(w, h);
    float px = (fx - 0.5f * w) * k, py = (fy - 0.5f * h) * k;
    o = v3p(pp.origin) + v3p(pp.right) * px + v3p(pp.up) * py;
    d = normalize(v3p(pp.forward));
    return;
  }
  if(G && pp.camera == CAMERA_THIN_LENS) {
    // ThinLensCamera::sample_ray_importance, get_focus_point, sample_lens_point
    // (thin_lens_camera.cpp:15-33,100-114)
    float k = pp.proj_dim / fmaxf(w, h);
    float px = (fx - 0.5f * w) * k, py = (fy - 0.5f * h) * k;
    V3 focus = v3(px * pp.focal_distance, py * pp.focal_distance, pp.focal_distance);
    Rand4 r = rand4(pp.seed, pixel, sample, kBlockCamera);
    float lx, ly;
    uniform_disk_sample(r.c, r.d, lx, ly);
    V3 R = v3p(pp.right), U = v3p(pp.up), F = v3p(pp.forward), O = v3p(pp.origin);
    V3 wf = O + R * focus.x + U * focus.y + F * focus.z;
    V3 wl = O + R * (lx * pp.lens_radius) + U * (ly * pp.lens_radius);
    o = wl;
    d = normalize(wf - wl);
    return;
  }
  // PinholeCamera::sample_ray_importance (pinhole_camera.cpp:13-31)
  float cx = fx / w - 0.5f, cy = fy / h - 0.5f;
  float nx, ny;
  if(w > h) { nx = cx; ny = cy * h / w; } else { nx = cx * w / h; ny = cy; }
  float px = nx * pp.proj_dim, py = ny * pp.proj_dim;
  V3 dir = v3p(pp.right) * px + v3p(pp.up) * py + v3p(pp.forward);
  d = normalize(dir);
  o = v3p(pp.origin);
}

// Direct lighting from one light (estimate_direct, path_renderer.cpp:135-206).
template<bool G>
DG_HD V3 estimate_direct(const PtScene& sc, const PtParams& pp, uint32_t li,
                         const SurfaceHit& g, const DevMaterial& m, V3 wo,
                         float u_bsdf, float v_bsdf, float c_bsdf, float u_l, float v_l,
                         uint32_t& rays) {
  const uint32_t req = F_ALL & ~F_DELTA;
  const DevLight& l = sc.lights[li];
  // the BSDF strategy only for area and background lights (:138-140)
  bool use_bsdf = pp.strategy != 2 && (light_is_area(l) || light_is_background(l));
  bool use_light = pp.strategy != 1;
  V3 sum = v3(0.f, 0.f, 0.f);
  if(use_bsdf) {
    BsdfSample bs = bsdf_sample<G>(m, g.frame, wo, req, u_bsdf, v_bsdf, c_bsdf);
    if(!(bs.pdf == 0.f || is_black(bs.f))) {
      // A background light counts only if the ray escapes, so whether anything
      // is hit is all that matters: an any-hit query gives the same answer.
      bool area = light_is_area(l);
      Hit h = area ? scene_trace<false, G>(sc, g.p, g.eps, bs.w, INFINITY)
                   : scene_trace<true, G>(sc, g.p, g.eps, bs.w, INFINITY);
      rays += 1;
      V3 L = v3(0.f, 0.f, 0.f);
      if(area) {
        L = area_light_hit_radiance<G>(sc, li, h, g.p, bs.w);
      } else if(h.prim == kMiss) {
        L = background_radiance(sc, l, bs.w);
      }
      if(!is_black(L)) {
        float w = 1.f;
        if(use_light) {
          float lp = light_pivot_pdf<G>(sc, l, bs.w, g.p);
          w = bs.pdf / (bs.pdf + lp);
        }
        sum = sum + bs.f * L * (w * fabsf(dot(g.n, bs.w)) / bs.pdf);
      }
    }
  }
  if(use_light) {
    LightSample ls = light_sample<G>(sc, l, g.p, g.eps, u_l, v_l);
    if(!(ls.pdf == 0.f || is_black(ls.L))) {
      V3 f = bsdf_eval<G>(m, g.frame, ls.wi, wo, req);
      if(!is_black(f)) {
        Hit h = scene_trace<true, G>(sc, ls.o, ls.tmin, ls.d, ls.tmax);
        rays += 1;
        if(h.prim == kMiss) {
          float w = 1.f;
          if(use_bsdf) {
            float bp = bsdf_pdf<G>(m, g.frame, ls.wi, wo, req);
            w = ls.pdf / (ls.pdf + bp);
          }
          sum = sum + f * ls.L * (w * fabsf(dot(g.n, ls.wi)) / ls.pdf);
        }
      }
    }
  }
  return sum;
}

// PathRenderer::sample (path_renderer.cpp:23-111) for one film position.
template<class Tape, bool G>
DG_HD PathResult pt_sample(const PtScene& sc, const PtParams& pp, uint32_t pixel,
                           uint32_t sample, float fx, float fy, Tape& tape) {
  PathResult res;
  res.rays = 0;
  V3 o, d;
  camera_ray<G>(pp, pixel, sample, fx, fy, o, d);
  float tmin = 0.f;
  V3 sum = v3(0.f, 0.f, 0.f);
  V3 thr = v3(1.f, 1.f, 1.f);
  uint32_t bounces = 0;
  bool last_delta = false;
  const uint32_t req_nd = F_ALL & ~F_DELTA;
  for(;;) {
    Hit h = scene_trace<false, G>(sc, o, tmin, d, INFINITY);
    res.rays += 1;
    bool hit = h.prim != kMiss;
    SurfaceHit g;
    if(hit) { g = surface_at<G>(sc, h, o, d); }
    if((bounces == 0 || last_delta) && bounces >= pp.min_depth && bounces <= pp.max_depth) {
      if(hit) {
        if(g.light) {
          const DevLight& l = sc.lights[g.light - 1];
          V3 Le = area_eval_radiance(sc, l, g.p, g.n, o);
          tape.emission(g.tri, thr, Le);
          sum = sum + thr * Le;
        }
      } else {
        for(uint32_t k = 0; k < sc.bg_count; ++k) {
          V3 c = thr * background_radiance(sc, sc.lights[sc.bg_light[k]], d);
          tape.background(c);
          sum = sum + c;
        }
      }
    }
    bounces += 1;
    if(!hit || bounces > pp.max_depth) { break; }

    V3 wo = normalize(-d);
    DevMaterial m = material_at(sc, g);
    uint32_t blk = bounce_block(bounces);
    Rand4 r0 = rand4(pp.seed, pixel, sample, blk);
    Rand4 r1 = rand4(pp.seed, pixel, sample, blk + 1);
    Rand4 r2 = rand4(pp.seed, pixel, sample, blk + 2);

    tape.vertex(g.tri, m);
    if(bounces >= pp.min_depth && bxdf_matches(m.bxdf_flags, req_nd)) {
      // sample_direct_lighting (path_renderer.cpp:113-132)
      if(pp.sample_all_lights) {
        for(uint32_t li = 0; li < sc.light_count; ++li) {
          uint32_t b2 = all_lights_block(bounces, li, sc.light_count);
          Rand4 a = rand4(pp.seed, pixel, sample, b2);
          Rand4 b = rand4(pp.seed, pixel, sample, b2 + 1);
          const DevLight& l = sc.lights[li];
          V3 c = estimate_direct<G>(sc, pp, li, g, m, wo, a.a, a.b, a.c, b.a, b.b, res.rays) * thr;
          tape.direct(l.kind == LIGHT_TRI ? l.tri : kMiss, c);
          sum = sum + c;
        }
      } else if(sc.light_count > 0) {
        uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, r0.a);
        float lpdf = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
        if(lpdf != 0.f) {
          const DevLight& l = sc.lights[li];
          V3 e = estimate_direct<G>(sc, pp, li, g, m, wo, r0.b, r0.c, r0.d, r1.a, r1.b, res.rays);
          V3 c = e * (1.f / lpdf) * thr;
          tape.direct(l.kind == LIGHT_TRI ? l.tri : kMiss, c);
          sum = sum + c;
        }
      }
    }

    uint32_t req = (pp.only_direct || bounces == pp.max_depth) ? (F_MODES | F_DELTA) : F_ALL;
    BsdfSample bs = bsdf_sample<G>(m, g.frame, wo, req, r1.c, r1.d, r2.a);
    if(is_black(bs.f) || bs.pdf == 0.f) { break; }
    V3 contrib = bs.f * (fabsf(dot(bs.w, g.n)) / bs.pdf);
    last_delta = (bs.flags & F_DELTA) != 0;
    thr = thr * contrib;
    if(bounces == pp.max_depth && !last_delta) {
      break;
    } else if(bounces >= 2 && bounces > pp.min_depth && pp.roulette) {
      float survive = clampf(average(contrib), 0.1f, 0.99f);
      if(r2.b > survive) { break; }
      thr = thr * (1.f / survive);
    }
    o = g.p;
    d = bs.w;
    tmin = g.eps;
  }
  // importance / ray_pdf of the pinhole camera is 1
  res.L = sum;
  return res;
}

}  // namespace dort_gpu
