// One path sample of the reference's "pt" renderer, for the device (and, for
// checking without a GPU, the host).
//
// Restates PathRenderer::sample / sample_direct_lighting / estimate_direct*
// (src/dort/path_renderer.cpp:23-206) over the flat device scene:
//   - BSDF: Bsdf (bsdf.cpp:50-242) specialised to the single BxDF that every
//     material in scope adds -- LambertBrdf (lambert_material.cpp:5-35),
//     MirrorBrdf (mirror_material.cpp:5-29), DielectricBxdf
//     (dielectric_material.cpp:32-116, fresnel.cpp:5-47), PhongBrdf
//     (phong_material.cpp:6-106) and a GGX conductor built on the reference's
//     GGX distribution (microfacet.cpp:19-86; the conductor itself has no
//     reference counterpart);
//   - lights: DiffuseLight on a triangle (diffuse_light.cpp:40-111,
//     shape.cpp:4-26, triangle.cpp:62-80), InfiniteLight
//     (infinite_light.cpp:5-65), EnvironmentLight (environment_light.cpp);
//   - camera: PinholeCamera::sample_ray_importance (pinhole_camera.cpp:13-31);
//   - light choice: DiscreteDistrib1d over approximate powers
//     (discrete_distrib_1d.cpp, scene.cpp:20-28).
// Random numbers come from Philox keyed by (seed, pixel, sample, block); see
// philox.cuh for the dimension layout.
#pragma once
#include <cmath>

#include "philox.cuh"
#include "pt_scene.h"
#include "trace.cuh"

namespace dort_gpu {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr float kInvFourPi = 0.07957747154594766788f;

struct V3 { float x, y, z; };
DG_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
DG_HD V3 v3p(const float* p) { return v3(p[0], p[1], p[2]); }
DG_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
DG_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
DG_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
DG_HD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
DG_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
DG_HD V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
DG_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DG_HD V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
DG_HD float length_sq(V3 a) { return dot(a, a); }
DG_HD float length(V3 a) { return sqrtf(length_sq(a)); }
DG_HD V3 normalize(V3 a) { return a * (1.f / length(a)); }
DG_HD bool is_black(V3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
DG_HD float average(V3 a) { return (1.f / 3.f) * (a.x + a.y + a.z); }
DG_HD float sq(float a) { return a * a; }
DG_HD float clampf(float v, float lo, float hi) { return v > hi ? hi : (v < lo ? lo : v); }

// geometry.cpp:4-11
DG_HD void coordinate_system(V3 v0, V3& v1, V3& v2) {
  if(fabsf(v0.x) > fabsf(v0.y)) {
    v1 = normalize(v3(-v0.z, 0.f, v0.x));
  } else {
    v1 = normalize(v3(0.f, -v0.z, v0.y));
  }
  v2 = cross(v0, v1);
}

// monte_carlo.cpp
DG_HD V3 cosine_hemisphere_sample(float u1, float u2) {
  float r = sqrtf(u1);
  float th = kTwoPi * u2;
  float x = cosf(th) * r, y = sinf(th) * r;
  float z = sqrtf(fmaxf(0.f, 1.f - x * x - y * y));
  return v3(x, y, z);
}
DG_HD float cosine_hemisphere_pdf(float cos_theta) { return fabsf(cos_theta * kInvPi); }
DG_HD V3 uniform_sphere_sample(float u1, float u2) {
  float z = 1.f - 2.f * u1;
  float r = sqrtf(fmaxf(0.f, 1.f - z * z));
  float phi = kTwoPi * u2;
  return v3(cosf(phi) * r, sinf(phi) * r, z);
}
DG_HD V3 power_cosine_hemisphere_sample(float u1, float u2, float e) {
  float phi = kTwoPi * u1;
  float ct = powf(u2, 1.f / (1.f + e));
  float st = sqrtf(1.f - ct * ct);
  return v3(cosf(phi) * st, sinf(phi) * st, ct);
}
DG_HD float power_cosine_hemisphere_pdf(float ct, float e) {
  return (e + 1.f) * powf(ct, e) * kInvTwoPi;
}

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
  float sp = sinf(u2 * kTwoPi), cp = cosf(u2 * kTwoPi);
  V3 m = v3(st * sp, st * cp, ct);
  pdf = ggx_d(m, alpha) * ct;
  return m;
}
DG_HD V3 schlick(V3 f0, float cos_i) {
  float k = powf(1.f - fminf(fabsf(cos_i), 1.f), 5.f);
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

// Bxdf::eval_f for the resolved BxDF of `m` (local directions).
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
    default:
      return v3(0.f, 0.f, 0.f);   // mirror, dielectric: delta only
  }
}

// Bxdf light_f_pdf / symmetric_f_pdf (local directions).
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
    case DORT_MAT_DIELECTRIC: {
      // dielectric_material.cpp:33-99 with fix_is_light = false, not thin
      bool s_refl = request & F_REFL, s_trans = request & F_TRANS;
      float ir, it;
      if(wf.z >= 0.f) { ir = 1.f; it = m.p0; } else { ir = m.p0; it = 1.f; }
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
      float r = fr, t = 1.f - r;
      bool reflect = uc <= r && s_refl;
      bool transmit = uc > r && s_trans;
      float rp = s_trans ? r : 1.f;
      float tp = s_refl ? t : 1.f;
      if(reflect) {
        flags = F_DELTA | F_REFL;
        pdf = rp;
        wg = w_reflect;
        return v3p(m.c) * (r / cr);
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
      pdf = bxdf_pdf(m, wg, wf, request);
      return bxdf_eval(m, wg, wf, request);
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
  V3 f = bxdf_sample(m, wf, request, u, v, uc, wg, pdf, flags);
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
DG_HD V3 bsdf_eval(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo, uint32_t request) {
  V3 wi_l = fr.to_local(wi), wo_l = fr.to_local(wo);
  bool reflection = wo_l.z * wi_l.z > 0.f;
  uint32_t er = request & ((F_LOBES & ~F_DELTA) | (reflection ? F_REFL : F_TRANS));
  if(!(er & F_MODES)) { return v3(0.f, 0.f, 0.f); }
  if(!bxdf_matches(m.bxdf_flags, er)) { return v3(0.f, 0.f, 0.f); }
  V3 f = bxdf_eval(m, wi_l, wo_l, er);
  float dn = fabsf(dot(fr.n, wi));
  return (dn * dn == 0.f) ? v3(0.f, 0.f, 0.f) : f;
}

// Bsdf::light_f_pdf (bsdf.cpp:194-225).
DG_HD float bsdf_pdf(const DevMaterial& m, const Frame& fr, V3 wi, V3 wo, uint32_t request) {
  if(!bxdf_matches(m.bxdf_flags, request)) { return 0.f; }
  return bxdf_pdf(m, fr.to_local(wi), fr.to_local(wo), request);
}

// ---- scene access ---------------------------------------------------------------

struct SurfaceHit {
  V3 p, n;          // point, unit geometric normal (cross(e2, e1))
  Frame frame;
  float eps;        // ray epsilon |1e-3 t|
  uint32_t tri;
  uint32_t mat;
  uint32_t light;   // light index + 1, 0 if not emissive
};

DG_HD SurfaceHit surface_at(const PtScene& sc, const Hit& h) {
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
  if(sc.tri_albedo && m.bxdf_flags) {
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
  float theta = dv * kPi;
  float phi = (du - 0.5f) * kTwoPi;
  float ct = cosf(theta), st = sinf(theta), cp = cosf(phi), sp = sinf(phi);
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
// PiecewiseDistrib2d::sample_cdf_slice (piecewise_distrib_2d.cpp:47-70)
DG_HD float env_sample_slice(const float* cdf, uint32_t n_plus_1, float u, uint32_t& idx) {
  uint32_t begin = 0, end = n_plus_1 - 1;
  while(begin + 1 < end) {
    uint32_t mid = begin + (end - begin) / 2;
    if(DG_LDG(cdf + mid) < u) { begin = mid; } else { end = mid; }
  }
  float c0 = DG_LDG(cdf + begin), c1 = DG_LDG(cdf + begin + 1);
  idx = begin;
  return float(begin) + (u - c0) / (c1 - c0);
}
DG_HD V3 env_sample_dir(const DevEnv& e, float u, float v, float& du, float& dv, float& pdf) {
  uint32_t yi, xi;
  float y = env_sample_slice(e.marginal_cdf, e.h + 1, v, yi);
  float x = env_sample_slice(e.cond_cdf + size_t(e.w + 1) * yi, e.w + 1, u, xi);
  du = x / float(e.w);
  dv = y / float(e.h);
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

// Light::pivot_radiance_pdf
DG_HD float light_pivot_pdf(const PtScene& sc, const DevLight& l, V3 wi, V3 pivot) {
  if(l.kind == LIGHT_INFINITE) { return kInvFourPi; }
  if(l.kind == LIGHT_ENV) { return env_dir_pdf(sc.env, wi); }
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
};

// Light::sample_pivot_radiance for the three light kinds.
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

DG_HD void camera_ray(const PtParams& pp, float fx, float fy, V3& o, V3& d) {
  // PinholeCamera::sample_ray_importance (pinhole_camera.cpp:13-31)
  float w = float(pp.width), h = float(pp.height);
  float cx = fx / w - 0.5f, cy = fy / h - 0.5f;
  float nx, ny;
  if(w > h) { nx = cx; ny = cy * h / w; } else { nx = cx * w / h; ny = cy; }
  float px = nx * pp.proj_dim, py = ny * pp.proj_dim;
  V3 dir = v3p(pp.right) * px + v3p(pp.up) * py + v3p(pp.forward);
  d = normalize(dir);
  o = v3p(pp.origin);
}

// Direct lighting from one light (estimate_direct, path_renderer.cpp:135-206).
DG_HD V3 estimate_direct(const PtScene& sc, const PtParams& pp, const DevLight& l,
                         const SurfaceHit& g, const DevMaterial& m, V3 wo,
                         float u_bsdf, float v_bsdf, float c_bsdf, float u_l, float v_l,
                         uint32_t& rays) {
  const uint32_t req = F_ALL & ~F_DELTA;
  bool use_bsdf = pp.strategy != 2;   // area and background lights only; no delta lights
  bool use_light = pp.strategy != 1;
  V3 sum = v3(0.f, 0.f, 0.f);
  if(use_bsdf) {
    BsdfSample bs = bsdf_sample(m, g.frame, wo, req, u_bsdf, v_bsdf, c_bsdf);
    if(!(bs.pdf == 0.f || is_black(bs.f))) {
      // A background light counts only if the ray escapes, so whether anything
      // is hit is all that matters: an any-hit query gives the same answer.
      Hit h = l.kind == LIGHT_TRI
          ? trace_ray<false, false>(sc.trace, g.p.x, g.p.y, g.p.z, g.eps, bs.w.x, bs.w.y, bs.w.z,
                             INFINITY)
          : trace_ray<true, false>(sc.trace, g.p.x, g.p.y, g.p.z, g.eps, bs.w.x, bs.w.y, bs.w.z,
                            INFINITY);
      rays += 1;
      V3 L = v3(0.f, 0.f, 0.f);
      if(h.prim != kMiss && l.kind == LIGHT_TRI) {
        if(h.prim == l.tri) {
          const float4* sh = sc.shade + 3 * size_t(h.prim);
          float4 a = DG_LDG(sh), b = DG_LDG(sh + 1), c = DG_LDG(sh + 2);
          V3 p0 = v3(a.x, a.y, a.z), p1 = v3(b.x, b.y, b.z), p2 = v3(c.x, c.y, c.z);
          float b0 = 1.f - h.b1 - h.b2;
          V3 lp = b0 * p0 + h.b1 * p1 + h.b2 * p2;
          V3 ln = normalize(cross(p2 - p0, p1 - p0));
          L = area_eval_radiance(sc, l, lp, ln, g.p);
        }
      } else if(h.prim == kMiss && l.kind != LIGHT_TRI) {
        L = background_radiance(sc, l, bs.w);
      }
      if(!is_black(L)) {
        float w = 1.f;
        if(use_light) {
          float lp = light_pivot_pdf(sc, l, bs.w, g.p);
          w = bs.pdf / (bs.pdf + lp);
        }
        sum = sum + bs.f * L * (w * fabsf(dot(g.n, bs.w)) / bs.pdf);
      }
    }
  }
  if(use_light) {
    LightSample ls = light_sample(sc, l, g.p, g.eps, u_l, v_l);
    if(!(ls.pdf == 0.f || is_black(ls.L))) {
      V3 f = bsdf_eval(m, g.frame, ls.wi, wo, req);
      if(!is_black(f)) {
        Hit h = trace_ray<true, false>(sc.trace, ls.o.x, ls.o.y, ls.o.z, ls.tmin, ls.d.x, ls.d.y,
                                ls.d.z, ls.tmax);
        rays += 1;
        if(h.prim == kMiss) {
          float w = 1.f;
          if(use_bsdf) {
            float bp = bsdf_pdf(m, g.frame, ls.wi, wo, req);
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
template<class Tape>
DG_HD PathResult pt_sample(const PtScene& sc, const PtParams& pp, uint32_t pixel,
                           uint32_t sample, float fx, float fy, Tape& tape) {
  PathResult res;
  res.rays = 0;
  V3 o, d;
  camera_ray(pp, fx, fy, o, d);
  float tmin = 0.f;
  V3 sum = v3(0.f, 0.f, 0.f);
  V3 thr = v3(1.f, 1.f, 1.f);
  uint32_t bounces = 0;
  bool last_delta = false;
  const uint32_t req_nd = F_ALL & ~F_DELTA;
  for(;;) {
    Hit h = trace_ray<false, false>(sc.trace, o.x, o.y, o.z, tmin, d.x, d.y, d.z, INFINITY);
    res.rays += 1;
    bool hit = h.prim != kMiss;
    SurfaceHit g;
    if(hit) { g = surface_at(sc, h); }
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
          V3 c = estimate_direct(sc, pp, l, g, m, wo, a.a, a.b, a.c, b.a, b.b, res.rays) * thr;
          tape.direct(l.kind == LIGHT_TRI ? l.tri : kMiss, c);
          sum = sum + c;
        }
      } else if(sc.light_count > 0) {
        uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, r0.a);
        float lpdf = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
        if(lpdf != 0.f) {
          const DevLight& l = sc.lights[li];
          V3 e = estimate_direct(sc, pp, l, g, m, wo, r0.b, r0.c, r0.d, r1.a, r1.b, res.rays);
          V3 c = e * (1.f / lpdf) * thr;
          tape.direct(l.kind == LIGHT_TRI ? l.tri : kMiss, c);
          sum = sum + c;
        }
      }
    }

    uint32_t req = (pp.only_direct || bounces == pp.max_depth) ? (F_MODES | F_DELTA) : F_ALL;
    BsdfSample bs = bsdf_sample(m, g.frame, wo, req, r1.c, r1.d, r2.a);
    if(is_black(bs.f) || bs.pdf == 0.f) { break; }
    V3 contrib = bs.f * (fabsf(dot(bs.w, g.n)) / bs.pdf);
    last_delta = (bs.flags & F_DELTA) != 0;
    thr = thr * contrib;
    if(bounces == pp.max_depth && !last_delta) {
      break;
    } else if(bounces >= 2 && bounces > pp.min_depth) {
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
