// Host-side scene assembly (see scene_build.h).
//
// Follows what the reference's builder and lights compute before rendering:
//   - materials resolve to the single BxDF their add_bxdfs would add
//     (lambert_material.cpp:27-35, mirror_material.cpp:24-29,
//     dielectric_material.cpp:105-116, phong_material.cpp:98-106);
//   - every emissive triangle and every emissive analytic shape becomes one
//     DiffuseLight (diffuse_light.cpp), then the delta lights (PointLight,
//     DirectionalLight) in the caller's order, then the background lights in
//     the order InfiniteLight, EnvironmentLight;
//   - the scene bounds are the union of the triangles' boxes and the shapes'
//     boxes taken through their transforms (Transform::apply(Box),
//     transform.cpp:27-40);
//   - the light choice CDF is DiscreteDistrib1d over approximate_power()
//     averages (scene.cpp:20-28, discrete_distrib_1d.cpp:4-20), with the
//     scene radius of build_scene (lua_builder.cpp:124-126);
//   - the environment map's 2-D distribution is PiecewiseDistrib2d over
//     |average(texel) * clamp(cos theta, 0, 1)| (environment_light.cpp:6-30,
//     piecewise_distrib_2d.cpp:4-35).
#include "scene_build.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace dort_gpu {
namespace {

struct F3 { float x, y, z; };
F3 f3(const float* p) { return {p[0], p[1], p[2]}; }
F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 crs(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float dt(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float len(F3 a) { return std::sqrt(dt(a, a)); }
F3 nrm(F3 a) { float k = 1.f / len(a); return {a.x * k, a.y * k, a.z * k}; }
float avg3(const float* c) { return (1.f / 3.f) * (c[0] + c[1] + c[2]); }
bool black3(const float* c) { return c[0] == 0.f && c[1] == 0.f && c[2] == 0.f; }

bool resolve_material(const dort_material& in, DevMaterial& m, std::string& err) {
  std::memset(&m, 0, sizeof(m));
  m.kind = in.kind;
  for(int i = 0; i < 3; ++i) { m.c[i] = in.color[i]; m.c2[i] = in.color2[i]; }
  for(int i = 0; i < 3; ++i) {
    if(!std::isfinite(in.color[i]) || !std::isfinite(in.color2[i]) ||
       in.color[i] < 0.f || in.color2[i] < 0.f) {
      err = "material colors must be finite and non-negative";
      return false;
    }
  }
  switch(in.kind) {
    case DORT_MAT_LAMBERT:
      m.bxdf_flags = black3(m.c) ? 0 : (F_REFL | F_DIFF);
      return true;
    case DORT_MAT_MIRROR:
      m.bxdf_flags = black3(m.c) ? 0 : (F_DELTA | F_REFL);
      return true;
    case DORT_MAT_DIELECTRIC: {
      // param[0] = ior_inside (0: 1.5), param[1] = ior_outside (0: 1),
      // param[2] != 0: thin; DielectricMaterial::add_bxdfs adds nothing for a
      // non-positive ior or black tints (dielectric_material.cpp:105-116)
      float ior_in = in.param[0] != 0.f ? in.param[0] : 1.5f;
      float ior_out = in.param[1] != 0.f ? in.param[1] : 1.f;
      m.p0 = ior_in;
      m.p1 = ior_out;
      m.p2 = in.param[2] != 0.f ? 1.f : 0.f;
      bool none = (black3(m.c) && black3(m.c2)) || !(ior_in > 0.f) || !(ior_out > 0.f);
      m.bxdf_flags = none ? 0 : (F_DELTA | F_REFL | F_TRANS);
      return true;
    }
    case DORT_MAT_OREN_NAYAR: {
      // OrenNayarMaterial::add_bxdfs (oren_nayar_material.cpp:60-71): Lambert
      // for sigma = 0; A and B of OrenNayarBrdf::eval_f (:9-11)
      float sigma = in.param[0];
      if(!std::isfinite(sigma)) { err = "oren_nayar sigma must be finite"; return false; }
      if(black3(m.c)) {
        m.bxdf_flags = 0;
      } else if(sigma == 0.f) {
        m.kind = DORT_MAT_LAMBERT;
        m.bxdf_flags = F_REFL | F_DIFF;
      } else {
        float s2 = sigma * sigma;
        m.p0 = sigma;
        m.p1 = 1.f - 0.5f * s2 / (s2 + 0.33f);
        m.p2 = 0.45f * s2 / (s2 + 0.09f);
        m.bxdf_flags = F_REFL | F_DIFF;
      }
      return true;
    }
    case DORT_MAT_PHONG: {
      float s[3] = {m.c[0] + m.c2[0], m.c[1] + m.c2[1], m.c[2] + m.c2[2]};
      float mx = std::max(s[0], std::max(s[1], s[2]));
      if(mx > 1.f) {
        float darken = 1.f / mx;
        for(int i = 0; i < 3; ++i) { m.c[i] *= darken; m.c2[i] *= darken; }
      }
      m.p0 = in.param[0];
      if(!black3(m.c2)) {
        float dw = avg3(m.c), gw = avg3(m.c2);
        float sum = dw + gw;
        m.p1 = sum != 0.f ? gw / sum : 0.f;
        m.bxdf_flags = F_REFL | F_DIFF | F_GLOSSY;
      } else if(!black3(m.c)) {
        m.kind = DORT_MAT_LAMBERT;
        m.bxdf_flags = F_REFL | F_DIFF;
      } else {
        m.bxdf_flags = 0;
      }
      return true;
    }
    case DORT_MAT_CONDUCTOR:
      m.p0 = std::max(in.param[0], 1e-3f);
      m.bxdf_flags = black3(m.c) ? 0 : (F_REFL | F_GLOSSY);
      return true;
    default:
      err = "unknown material kind " + std::to_string(in.kind);
      return false;
  }
}

// DiscreteDistrib1d (discrete_distrib_1d.cpp:4-20)
std::vector<float> make_cdf(const std::vector<float>& xs) {
  std::vector<float> cdf;
  float sum = 0.f;
  for(float x : xs) { cdf.push_back(sum); sum += x; }
  cdf.push_back(sum);
  float inv = sum == 0.f ? 0.f : 1.f / sum;
  for(float& c : cdf) { c *= inv; }
  return cdf;
}

// Inverse of a 3x4 affine transform; false if singular.
bool invert_affine(const float* m, float* inv) {
  double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9],
         i = m[10];
  double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  double det = a * A + b * B + c * C;
  if(!(std::fabs(det) > 1e-30) || !std::isfinite(det)) { return false; }
  double r[9] = {A, -(b * i - c * h), b * f - c * e,
                 B, a * i - c * g, -(a * f - c * d),
                 C, -(a * h - b * g), a * e - b * d};
  for(int k = 0; k < 9; ++k) { r[k] /= det; }
  double t[3] = {m[3], m[7], m[11]};
  for(int row = 0; row < 3; ++row) {
    inv[4 * row] = float(r[3 * row]);
    inv[4 * row + 1] = float(r[3 * row + 1]);
    inv[4 * row + 2] = float(r[3 * row + 2]);
    inv[4 * row + 3] = float(-(r[3 * row] * t[0] + r[3 * row + 1] * t[1] + r[3 * row + 2] * t[2]));
  }
  return true;
}

// Shape-space bounding box (the shapes' bounds()).
void shape_local_bounds(const DevShape& s, float lo[3], float hi[3]) {
  switch(s.kind) {
    case SHAPE_SPHERE:
      for(int a = 0; a < 3; ++a) { lo[a] = -s.r; hi[a] = s.r; }
      break;
    case SHAPE_DISK:
      lo[0] = lo[1] = -s.r; hi[0] = hi[1] = s.r; lo[2] = hi[2] = s.z0;
      break;
    case SHAPE_CUBE:
      for(int a = 0; a < 3; ++a) { lo[a] = -1.f; hi[a] = 1.f; }
      break;
    default:   // cylinder
      lo[0] = lo[1] = -s.r; hi[0] = hi[1] = s.r; lo[2] = s.z0; hi[2] = s.z1;
      break;
  }
}

}  // namespace

// Alias table (Vose's method: M. D. Vose, "A Linear Algorithm for Generating
// Random Numbers with a Given Distribution", IEEE TSE 17(9), 1991) of the
// weights w[0..n): entry i = (probability of keeping i, the other index);
// picking i uniformly and keeping it with that probability, else taking its
// alias, draws index k with probability w[k] / sum(w).  Weights that sum to
// zero give every entry probability 1 (the table is then never used).
static void build_alias(const double* w, uint32_t n, float2* out) {
  double sum = 0.0;
  for(uint32_t i = 0; i < n; ++i) { sum += w[i]; }
  std::vector<double> q(n);
  std::vector<uint32_t> small, large;
  for(uint32_t i = 0; i < n; ++i) {
    q[i] = sum > 0.0 ? w[i] * double(n) / sum : 1.0;
    (q[i] < 1.0 ? small : large).push_back(i);
  }
  for(uint32_t i = 0; i < n; ++i) {
    uint32_t self = i;
    float bits;
    std::memcpy(&bits, &self, 4);
    out[i] = make_float2(1.f, bits);
  }
  while(!small.empty() && !large.empty()) {
    uint32_t s = small.back(), l = large.back();
    small.pop_back();
    large.pop_back();
    float bits;
    std::memcpy(&bits, &l, 4);
    out[s] = make_float2(float(q[s]), bits);
    q[l] = (q[l] + q[s]) - 1.0;
    (q[l] < 1.0 ? small : large).push_back(l);
  }
}

bool material_to_device(const dort_material& in, DevMaterial& m, std::string& err) {
  return resolve_material(in, m, err);
}

bool build_host_scene(const dort_scene_desc* desc, HostScene& hs, std::string& err,
                      bool allow_device_bvh) {
  if(desc->struct_size != sizeof(dort_scene_desc)) {
    err = "dort_scene_desc.struct_size mismatch (ABI version)";
    return false;
  }
  if(desc->flags & ~DORT_SCENE_WATERTIGHT) {
    err = "unknown dort_scene_desc.flags bits";
    return false;
  }
  uint32_t n = desc->tri_count;
  if(n > 0 && (!desc->verts || !desc->tris)) {
    err = "verts and tris are required when tri_count > 0";
    return false;
  }
  if(n > (1u << 30)) { err = "tri_count exceeds 2^30"; return false; }
  if(desc->tri_material && (!desc->materials || desc->material_count == 0)) {
    err = "tri_material given without materials";
    return false;
  }

  alloc_checkpoint();
  // materials (material 0 is a white Lambert when none are given)
  hs.mats.clear();
  if(desc->materials && desc->material_count > 0) {
    for(uint32_t i = 0; i < desc->material_count; ++i) {
      DevMaterial m;
      if(!resolve_material(desc->materials[i], m, err)) { return false; }
      hs.mats.push_back(m);
    }
  } else {
    dort_material def;
    std::memset(&def, 0, sizeof(def));
    def.kind = DORT_MAT_LAMBERT;
    def.color[0] = def.color[1] = def.color[2] = 0.5f;
    DevMaterial m;
    resolve_material(def, m, err);
    hs.mats.push_back(m);
  }

  if(desc->bvh_build > DORT_BVH_BUILD_PLOC) {
    err = "bvh_build must be DORT_BVH_BUILD_DEFAULT, _HOST, _DEVICE or _PLOC";
    return false;
  }
  hs.device_bvh = allow_device_bvh && desc->bvh_build != DORT_BVH_BUILD_HOST;
  BuildOptions opts;
  opts.width = desc->bvh_width ? desc->bvh_width : 8;
  if(hs.device_bvh) {
    if(opts.width < 2 || opts.width > 8) {
      err = "bvh_width must be 2..8";
      return false;
    }
    if(!validate_mesh(desc->verts, desc->vert_count, desc->tris, n, err)) { return false; }
  } else {
    auto b0 = std::chrono::steady_clock::now();
    if(!build_wide_bvh(desc->verts, desc->vert_count, desc->tris, n, opts, hs.bvh, err)) {
      return false;
    }
    hs.bvh_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - b0)
                    .count();
  }

  // per-triangle shading records and area lights
  hs.shade.assign(3 * size_t(n), make_float4(0.f, 0.f, 0.f, 0.f));
  hs.lights.clear();
  std::vector<float> powers;
  hs.emissive_count = 0;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for(uint32_t t = 0; t < n; ++t) {
    const float* p[3];
    for(int k = 0; k < 3; ++k) {
      p[k] = desc->verts + 3 * size_t(desc->tris[3 * size_t(t) + k]);
      for(int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], p[k][a]);
        hi[a] = std::max(hi[a], p[k][a]);
      }
    }
    uint32_t mat = desc->tri_material ? desc->tri_material[t] : 0;
    if(mat >= hs.mats.size()) {
      err = "triangle " + std::to_string(t) + " has material " + std::to_string(mat) +
            " >= material_count";
      return false;
    }
    uint32_t light = 0;
    if(desc->tri_emission) {
      const float* le = desc->tri_emission + 3 * size_t(t);
      for(int a = 0; a < 3; ++a) {
        if(!std::isfinite(le[a]) || le[a] < 0.f) {
          err = "triangle emission must be finite and non-negative";
          return false;
        }
      }
      if(!black3(le)) {
        DevLight l;
        std::memset(&l, 0, sizeof(l));
        l.kind = LIGHT_TRI;
        l.tri = t;
        for(int a = 0; a < 3; ++a) { l.L[a] = le[a]; }
        // the light's own triangle when it differs from the primitive
        const float* lv = desc->tri_light_verts ? desc->tri_light_verts + 9 * size_t(t) : nullptr;
        for(int a = 0; lv && a < 9; ++a) {
          if(!std::isfinite(lv[a])) { err = "tri_light_verts must be finite"; return false; }
        }
        F3 p0 = lv ? f3(lv) : f3(p[0]);
        F3 e1 = sub(lv ? f3(lv + 3) : f3(p[1]), p0), e2 = sub(lv ? f3(lv + 6) : f3(p[2]), p0);
        l.area = 0.5f * len(crs(e1, e2));      // Triangle::area (triangle.cpp:56-60)
        F3 nn = nrm(crs(e2, e1));
        l.p0[0] = p0.x; l.p0[1] = p0.y; l.p0[2] = p0.z;
        l.e1[0] = e1.x; l.e1[1] = e1.y; l.e1[2] = e1.z;
        l.e2[0] = e2.x; l.e2[1] = e2.y; l.e2[2] = e2.z;
        l.nn[0] = nn.x; l.nn[1] = nn.y; l.nn[2] = nn.z;
        float pw[3] = {l.area * le[0], l.area * le[1], l.area * le[2]};
        powers.push_back(avg3(pw));
        hs.lights.push_back(l);
        light = uint32_t(hs.lights.size());
        hs.emissive_count += 1;
      }
    }
    uint32_t matbits, lightbits;
    std::memcpy(&matbits, &mat, 4);
    std::memcpy(&lightbits, &light, 4);
    float mf, lf;
    std::memcpy(&mf, &matbits, 4);
    std::memcpy(&lf, &lightbits, 4);
    hs.shade[3 * size_t(t)] = make_float4(p[0][0], p[0][1], p[0][2], mf);
    hs.shade[3 * size_t(t) + 1] = make_float4(p[1][0], p[1][1], p[1][2], lf);
    hs.shade[3 * size_t(t) + 2] = make_float4(p[2][0], p[2][1], p[2][2], 0.f);
  }
  // analytic shapes (ShapePrimitive) and their area lights
  hs.shapes.clear();
  hs.light_shapes.clear();
  hs.shape_base = n;
  if(desc->shape_count > 0 && !desc->shapes) { err = "shapes is NULL with shape_count > 0"; return false; }
  if(desc->shape_count > kMaxShapes) {
    err = "at most " + std::to_string(kMaxShapes) + " analytic shapes (they are tested as a list)";
    return false;
  }
  for(uint32_t k = 0; k < desc->shape_count; ++k) {
    const dort_shape& in = desc->shapes[k];
    DevShape sh;
    std::memset(&sh, 0, sizeof(sh));
    sh.kind = in.kind;
    if(in.kind < DORT_SHAPE_SPHERE || in.kind > DORT_SHAPE_CYLINDER) {
      err = "shape " + std::to_string(k) + " has unknown kind " + std::to_string(in.kind);
      return false;
    }
    if(in.material >= hs.mats.size()) {
      err = "shape " + std::to_string(k) + " has material >= material_count";
      return false;
    }
    sh.mat = in.material;
    for(int a = 0; a < 4; ++a) {
      if(!std::isfinite(in.param[a])) { err = "shape parameters must be finite"; return false; }
    }
    sh.r = in.param[0];
    sh.z0 = in.param[1];
    sh.z1 = in.param[2];
    if(in.kind != DORT_SHAPE_CUBE && !(sh.r > 0.f)) { err = "shape radius must be positive"; return false; }
    if(in.kind == DORT_SHAPE_CYLINDER && !(sh.z1 > sh.z0)) {
      err = "cylinder needs z_max > z_min";
      return false;
    }
    for(int a = 0; a < 12; ++a) {
      if(!std::isfinite(in.to_world[a])) { err = "shape transform must be finite"; return false; }
      sh.m[a] = in.to_world[a];
    }
    if(!invert_affine(sh.m, sh.inv)) {
      err = "shape " + std::to_string(k) + " has a singular transform";
      return false;
    }
    // Transform::apply(Box) (transform.cpp:27-40): centre and half extents
    float blo[3], bhi[3];
    shape_local_bounds(sh, blo, bhi);
    for(int row = 0; row < 3; ++row) {
      float mid = sh.m[4 * row + 3], rad = 0.f;
      for(int c = 0; c < 3; ++c) {
        mid += sh.m[4 * row + c] * 0.5f * (blo[c] + bhi[c]);
        rad += std::fabs(sh.m[4 * row + c] * 0.5f * (bhi[c] - blo[c]));
      }
      lo[row] = std::min(lo[row], mid - rad);
      hi[row] = std::max(hi[row], mid + rad);
    }
    for(int a = 0; a < 3; ++a) {
      if(!std::isfinite(in.emission[a]) || in.emission[a] < 0.f) {
        err = "shape emission must be finite and non-negative";
        return false;
      }
    }
    if(!black3(in.emission)) {
      if(in.kind != DORT_SHAPE_SPHERE && in.kind != DORT_SHAPE_DISK) {
        err = "only spheres and disks can be area lights";
        return false;
      }
      DevShape ls = sh;
      if(in.flags & DORT_SHAPE_LIGHT_TRANSFORM) {
        for(int a = 0; a < 12; ++a) {
          if(!std::isfinite(in.light_to_world[a])) {
            err = "shape light transform must be finite";
            return false;
          }
          ls.m[a] = in.light_to_world[a];
        }
        if(!invert_affine(ls.m, ls.inv)) {
          err = "shape " + std::to_string(k) + " has a singular light transform";
          return false;
        }
      }
      DevLight l;
      std::memset(&l, 0, sizeof(l));
      l.kind = LIGHT_SHAPE;
      l.tri = uint32_t(hs.light_shapes.size());
      for(int a = 0; a < 3; ++a) { l.L[a] = in.emission[a]; }
      // DiffuseLight: area = shape->area() in shape space; approximate_power
      // = area * radiance (diffuse_light.cpp:5-12,118-120)
      float r = sh.r;
      l.area = in.kind == DORT_SHAPE_SPHERE ? 4.f * 3.14159265358979323846f * r * r
                                            : 3.14159265358979323846f * r * r;
      float pw[3] = {l.area * l.L[0], l.area * l.L[1], l.area * l.L[2]};
      powers.push_back(avg3(pw));
      hs.lights.push_back(l);
      sh.light = uint32_t(hs.lights.size());
      ls.light = sh.light;
      hs.light_shapes.push_back(ls);
      hs.emissive_count += 1;
    }
    hs.shapes.push_back(sh);
  }

  // Scene::radius = bounds.radius() (box.hpp:36-38)
  bool any = n > 0 || desc->shape_count > 0;
  F3 ext = any ? F3{hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]} : F3{0.f, 0.f, 0.f};
  hs.radius = len(ext) * 0.5f;
  for(int a = 0; a < 3; ++a) { hs.centroid[a] = any ? 0.5f * (lo[a] + hi[a]) : 0.f; }
  float r2pi = 3.14159265358979323846f * hs.radius * hs.radius;

  // delta lights
  if(desc->light_count > 0 && !desc->lights) { err = "lights is NULL with light_count > 0"; return false; }
  for(uint32_t k = 0; k < desc->light_count; ++k) {
    const dort_light& in = desc->lights[k];
    for(int a = 0; a < 3; ++a) {
      if(!std::isfinite(in.rgb[a]) || in.rgb[a] < 0.f || !std::isfinite(in.vec[a])) {
        err = "delta light values must be finite (and colors non-negative)";
        return false;
      }
    }
    DevLight l;
    std::memset(&l, 0, sizeof(l));
    for(int a = 0; a < 3; ++a) { l.L[a] = in.rgb[a]; }
    float pw[3];
    if(in.kind == DORT_LIGHT_POINT) {
      // PointLight: approximate_power = 4 pi intensity (point_light.cpp:59-61)
      l.kind = LIGHT_POINT;
      for(int a = 0; a < 3; ++a) { l.p0[a] = in.vec[a]; pw[a] = 4.f * 3.14159265358979323846f * l.L[a]; }
    } else if(in.kind == DORT_LIGHT_DIRECTIONAL) {
      // DirectionalLight: normalized direction; approximate_power = pi r^2 L
      // (directional_light.cpp:5-12,66-68)
      F3 dir = f3(in.vec);
      if(!(len(dir) > 0.f)) { err = "directional light needs a non-zero direction"; return false; }
      dir = nrm(dir);
      l.kind = LIGHT_DIR;
      l.nn[0] = dir.x; l.nn[1] = dir.y; l.nn[2] = dir.z;
      for(int a = 0; a < 3; ++a) { pw[a] = r2pi * l.L[a]; }
    } else {
      err = "light " + std::to_string(k) + " has unknown kind " + std::to_string(in.kind);
      return false;
    }
    powers.push_back(avg3(pw));
    hs.lights.push_back(l);
  }

  hs.bg_count = 0;
  if(!black3(desc->sky_const)) {
    DevLight l;
    std::memset(&l, 0, sizeof(l));
    l.kind = LIGHT_INFINITE;
    for(int a = 0; a < 3; ++a) { l.L[a] = desc->sky_const[a]; }
    float pw[3] = {r2pi * l.L[0], r2pi * l.L[1], r2pi * l.L[2]};
    powers.push_back(avg3(pw));
    hs.lights.push_back(l);
    hs.bg_light[hs.bg_count++] = uint32_t(hs.lights.size() - 1);
  }
  hs.env_rgb.clear();
  std::memset(&hs.env, 0, sizeof(hs.env));
  if(desc->sky_rgb && desc->sky_width > 0 && desc->sky_height > 0) {
    uint32_t w = desc->sky_width, h = desc->sky_height;
    if(size_t(w) * h > (size_t(1) << 26)) { err = "sky image too large"; return false; }
    hs.env_rgb.assign(desc->sky_rgb, desc->sky_rgb + 3 * size_t(w) * h);
    for(float v : hs.env_rgb) {
      if(!std::isfinite(v) || v < 0.f) { err = "sky image must be finite and non-negative"; return false; }
    }
    float scale[3] = {1.f, 1.f, 1.f};
    if(!black3(desc->sky_scale)) { for(int a = 0; a < 3; ++a) { scale[a] = desc->sky_scale[a]; } }
    F3 up = black3(desc->sky_up) ? F3{0.f, 1.f, 0.f} : f3(desc->sky_up);
    F3 fwd = black3(desc->sky_fwd) ? F3{1.f, 0.f, 0.f} : f3(desc->sky_fwd);
    // EnvironmentLight constructor (environment_light.cpp:6-31)
    F3 upn = nrm(up);
    F3 tt = nrm(crs(up, fwd));
    F3 ss = crs(upn, tt);
    std::vector<float> values(size_t(w) * h);
    double vs[3] = {0, 0, 0};
    float vsum[3] = {0.f, 0.f, 0.f};
    float vweight = 0.f;
    (void)vs;
    for(uint32_t y = 0; y < h; ++y) {
      float theta = (float(y) + 0.5f) / float(h) * 3.14159265358979323846f;
      float ct = std::min(std::max(std::cos(theta), 0.f), 1.f);
      for(uint32_t x = 0; x < w; ++x) {
        const float* px = &hs.env_rgb[3 * (size_t(y) * w + x)];
        values[size_t(y) * w + x] = std::fabs(avg3(px) * ct);
        for(int a = 0; a < 3; ++a) { vsum[a] += px[a] * ct; }
        vweight += ct;
      }
    }
    // PiecewiseDistrib2d (piecewise_distrib_2d.cpp:4-35): texel probability
    // value / sum (its pdf over (u, v) is that times w * h); rows chosen by
    // their sums, columns within a row by their values
    hs.env_pdfs.assign(size_t(w) * h, 0.f);
    float sum = 0.f;
    for(uint32_t y = 0; y < h; ++y) {
      float ysum = 0.f;
      for(uint32_t x = 0; x < w; ++x) { ysum += values[size_t(y) * w + x]; }
      sum += ysum;
    }
    float inv_sum = 1.f / sum;
    for(size_t i = 0; i < values.size(); ++i) { hs.env_pdfs[i] = values[i] * inv_sum; }
    // the same row and column distributions as alias tables (O(1) sampling)
    std::vector<double> rw(h), cw(w);
    hs.env_row_alias.resize(h);
    hs.env_col_alias.resize(size_t(w) * h);
    for(uint32_t y = 0; y < h; ++y) {
      double rs = 0.0;
      for(uint32_t x = 0; x < w; ++x) {
        cw[x] = values[size_t(y) * w + x];
        rs += cw[x];
      }
      rw[y] = rs;
      build_alias(cw.data(), w, hs.env_col_alias.data() + size_t(y) * w);
    }
    build_alias(rw.data(), h, hs.env_row_alias.data());
    hs.env.w = w;
    hs.env.h = h;
    for(int a = 0; a < 3; ++a) { hs.env.scale[a] = scale[a]; }
    hs.env.up[0] = upn.x; hs.env.up[1] = upn.y; hs.env.up[2] = upn.z;
    hs.env.s[0] = ss.x; hs.env.s[1] = ss.y; hs.env.s[2] = ss.z;
    hs.env.t[0] = tt.x; hs.env.t[1] = tt.y; hs.env.t[2] = tt.z;
    DevLight l;
    std::memset(&l, 0, sizeof(l));
    l.kind = LIGHT_ENV;
    float ar[3];
    for(int a = 0; a < 3; ++a) { ar[a] = scale[a] * vsum[a] / vweight; }
    float pw[3] = {r2pi * ar[0], r2pi * ar[1], r2pi * ar[2]};
    powers.push_back(avg3(pw));
    hs.lights.push_back(l);
    hs.bg_light[hs.bg_count++] = uint32_t(hs.lights.size() - 1);
  }
  hs.light_cdf = make_cdf(powers);
  // features only the general instantiation of the path code handles
  hs.general = (!hs.shapes.empty() || desc->light_count > 0) ? 1u : 0u;
  for(const DevMaterial& m : hs.mats) {
    if(m.kind == DORT_MAT_OREN_NAYAR && m.bxdf_flags) { hs.general = 1u; }
    if(m.kind == DORT_MAT_DIELECTRIC && (m.p1 != 1.f || m.p2 != 0.f)) { hs.general = 1u; }
  }
  return true;
}

PtScene host_view(const HostScene& hs) {
  PtScene sc;
  std::memset(&sc, 0, sizeof(sc));
  sc.trace.nodes = reinterpret_cast<const uint4*>(traversal_nodes(hs.bvh));
  sc.trace.tris = reinterpret_cast<const float4*>(hs.bvh.tris.data());
  sc.trace.node_count = uint32_t(hs.bvh.nodes.size());
  sc.trace.tri_count = uint32_t(hs.bvh.tris.size());
  sc.shade = hs.shade.data();
  sc.mats = hs.mats.data();
  sc.mat_count = uint32_t(hs.mats.size());
  sc.lights = hs.lights.data();
  sc.light_count = uint32_t(hs.lights.size());
  sc.light_cdf = hs.light_cdf.data();
  sc.bg_count = hs.bg_count;
  sc.bg_light[0] = hs.bg_light[0];
  sc.bg_light[1] = hs.bg_light[1];
  sc.env = hs.env;
  sc.env.rgb = hs.env_rgb.empty() ? nullptr : hs.env_rgb.data();
  sc.env.pdfs = hs.env_pdfs.empty() ? nullptr : hs.env_pdfs.data();
  sc.env.row_alias = hs.env_row_alias.empty() ? nullptr : hs.env_row_alias.data();
  sc.env.col_alias = hs.env_col_alias.empty() ? nullptr : hs.env_col_alias.data();
  sc.shapes = hs.shapes.empty() ? nullptr : hs.shapes.data();
  sc.shape_count = uint32_t(hs.shapes.size());
  for(int a = 0; a < 3; ++a) { sc.centroid[a] = hs.centroid[a]; }
  sc.radius = hs.radius;
  sc.shape_base = hs.shape_base;
  sc.light_shapes = hs.light_shapes.empty() ? nullptr : hs.light_shapes.data();
  sc.general = hs.general;
  return sc;
}

}  // namespace dort_gpu
