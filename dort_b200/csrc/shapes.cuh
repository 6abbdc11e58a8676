// Analytic shapes of the reference placed by an affine transform, as
// ShapePrimitive does (primitive.cpp:28-58): the ray is taken into the
// shape's own space, intersected there, and the hit is brought back.
//   SphereShape    sphere_shape.cpp:10-147
//   DiskShape      disk_shape.cpp:4-78
//   CubeShape      cube_shape.cpp:4-97 ([-1, 1]^3)
//   CylinderShape  cylinder_shape.cpp:10-111 (no caps)
// plus the area-light sampling of spheres and disks (Shape::sample_point_pivot
// / point_pivot_pdf, shape.cpp:4-26, and the sphere's cone sampling).
#pragma once
#include "pt_math.cuh"
#include "pt_scene.h"

namespace dort_gpu {

// The shape code rounds every product and sum on its own (DG_MUL / DG_ADD /
// DG_SUB: no fused multiply-add), as the reference's float arithmetic does.
// Where a shape's face and a triangle coincide (a box standing on a floor)
// the hit found depends on that rounding.

DG_HD float dot3_rn(V3 a, V3 b) { return dot_rn(a.x, a.y, a.z, b.x, b.y, b.z); }
DG_HD V3 madd_rn(V3 o, V3 d, float t) {   // o + d t
  return v3(DG_ADD(o.x, DG_MUL(d.x, t)), DG_ADD(o.y, DG_MUL(d.y, t)),
            DG_ADD(o.z, DG_MUL(d.z, t)));
}

// 3x4 row-major affine transforms
DG_HD V3 xf_vec(const float* m, V3 v) {
  return v3(dot_rn(m[0], m[1], m[2], v.x, v.y, v.z), dot_rn(m[4], m[5], m[6], v.x, v.y, v.z),
            dot_rn(m[8], m[9], m[10], v.x, v.y, v.z));
}
DG_HD V3 xf_point(const float* m, V3 p) {
  V3 r = xf_vec(m, p);
  return v3(DG_ADD(r.x, m[3]), DG_ADD(r.y, m[7]), DG_ADD(r.z, m[11]));
}
// A shape-space normal taken to world space: the transpose of the inverse.
DG_HD V3 xf_normal(const float* inv, V3 n) {
  return v3(dot_rn(inv[0], inv[4], inv[8], n.x, n.y, n.z),
            dot_rn(inv[1], inv[5], inv[9], n.x, n.y, n.z),
            dot_rn(inv[2], inv[6], inv[10], n.x, n.y, n.z));
}

// math.cpp:21-38: the two roots of A x^2 + B x + C (false if none or one)
DG_HD bool solve_quadratic(float A, float B, float C, float& x1, float& x2) {
  float disc = DG_SUB(DG_MUL(B, B), DG_MUL(DG_MUL(4.f, A), C));
  if(disc <= 0.f) { return false; }
  float sd = sqrtf(disc);
  float q = B < 0.f ? DG_MUL(-0.5f, DG_SUB(B, sd)) : DG_MUL(-0.5f, DG_ADD(B, sd));
  x1 = q / A;
  x2 = C / q;
  return true;
}

DG_HD float v3_get(V3 v, uint32_t axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// Shape-space ray query.  Closest hit: the nearest surface crossing with t in
// [t_min, t_max] (the reference's hit), `face` = cube axis * 2 + (1 if the
// ray direction is negative on it).  Any hit: the reference's hit_p.
template<bool ANY_HIT>
DG_HD bool shape_hit(const DevShape& s, V3 o, V3 d, float t_min, float t_max, float& t_out,
                     uint32_t& face) {
  face = 0;
  switch(s.kind) {
    case SHAPE_SPHERE: {
      // SphereShape::solve_hit_t (sphere_shape.cpp:123-146)
      float a = dot3_rn(d, d), b = DG_MUL(2.f, dot3_rn(o, d));
      float c = DG_SUB(dot3_rn(o, o), DG_MUL(s.r, s.r));
      float t0, t1;
      if(!solve_quadratic(a, b, c, t0, t1)) { return false; }
      if(t1 < t0) { float x = t0; t0 = t1; t1 = x; }
      if(t_min <= t0 && t0 <= t_max) { t_out = t0; return true; }
      if(t_min <= t1 && t1 <= t_max) { t_out = t1; return true; }
      return false;
    }
    case SHAPE_DISK: {
      // DiskShape::hit / hit_p (disk_shape.cpp:5-56)
      if(d.z == 0.f) { return false; }
      float t = DG_SUB(s.z0, o.z) / d.z;
      if(!(t_min <= t && t <= t_max)) { return false; }
      float px = DG_ADD(o.x, DG_MUL(d.x, t)), py = DG_ADD(o.y, DG_MUL(d.y, t));
      if(DG_ADD(DG_MUL(px, px), DG_MUL(py, py)) > DG_MUL(s.r, s.r)) { return false; }
      t_out = t;
      return true;
    }
    case SHAPE_CUBE: {
      // CubeShape::hit / hit_p (cube_shape.cpp:4-97)
      float t0 = t_min, t1 = t_max;
      uint32_t ax0 = 3u, ax1 = 3u;
      bool neg0 = false, neg1 = false;
      for(uint32_t axis = 0; axis < 3; ++axis) {
        float inv = 1.f / v3_get(d, axis);
        float oa = v3_get(o, axis);
        float tn = DG_MUL(DG_SUB(-1.f, oa), inv), tf = DG_MUL(DG_SUB(1.f, oa), inv);
        bool negative = false;
        if(tn > tf) { float x = tn; tn = tf; tf = x; negative = true; }
        if(tn > t0) { t0 = tn; ax0 = axis; neg0 = negative; }
        if(tf < t1) { t1 = tf; ax1 = axis; neg1 = negative; }
        if(t0 > t1) { return false; }
      }
      if(ANY_HIT) { t_out = t0; return true; }
      if(ax0 != 3u) {
        t_out = t0;
        face = ax0 * 2u + (neg0 ? 1u : 0u);
      } else if(ax1 != 3u) {
        t_out = t1;
        face = ax1 * 2u + (neg1 ? 1u : 0u);
      } else {
        return false;
      }
      return true;
    }
    case SHAPE_CYLINDER: {
      // CylinderShape::solve_hit_t (cylinder_shape.cpp:75-110)
      float a = DG_ADD(DG_MUL(d.x, d.x), DG_MUL(d.y, d.y));
      float b = DG_MUL(2.f, DG_ADD(DG_MUL(o.x, d.x), DG_MUL(o.y, d.y)));
      float c = DG_SUB(DG_ADD(DG_MUL(o.x, o.x), DG_MUL(o.y, o.y)), DG_MUL(s.r, s.r));
      float t0, t1;
      if(!solve_quadratic(a, b, c, t0, t1)) { return false; }
      if(t1 < t0) { float x = t0; t0 = t1; t1 = x; }
      if(t_min <= t0 && t0 <= t_max) {
        float z = DG_ADD(o.z, DG_MUL(d.z, t0));
        if(s.z0 <= z && z <= s.z1) { t_out = t0; return true; }
      }
      if(t_min <= t1 && t1 <= t_max) {
        float z = DG_ADD(o.z, DG_MUL(d.z, t1));
        if(s.z0 <= z && z <= s.z1) { t_out = t1; return true; }
      }
      return false;
    }
    default:
      return false;
  }
}

// Shape-space geometric normal at shape-space point pl of a closest hit.
DG_HD V3 shape_local_normal(const DevShape& s, V3 pl, uint32_t face) {
  switch(s.kind) {
    case SHAPE_SPHERE: return pl * (1.f / s.r);
    case SHAPE_DISK: return v3(0.f, 0.f, 1.f);
    case SHAPE_CUBE: {
      // cube_shape.cpp:56: +axis when the ray runs towards -axis, else -axis
      float v = (face & 1u) ? 1.f : -1.f;
      uint32_t axis = face >> 1;
      return v3(axis == 0 ? v : 0.f, axis == 1 ? v : 0.f, axis == 2 ? v : 0.f);
    }
    case SHAPE_CYLINDER: return v3(pl.x, pl.y, 0.f) * (1.f / s.r);
    default: return v3(0.f, 0.f, 1.f);
  }
}

// Ray epsilon of a hit at parameter t (sphere 5e-3 |t|, cylinder 5e-3 |t|,
// disk and cube 1e-3 t).
DG_HD float shape_ray_epsilon(const DevShape& s, float t) {
  return (s.kind == SHAPE_SPHERE || s.kind == SHAPE_CYLINDER) ? 5e-3f * fabsf(t) : 1e-3f * t;
}

DG_HD float shape_area(const DevShape& s) {
  switch(s.kind) {
    case SHAPE_SPHERE: return 4.f * kPi * s.r * s.r;
    case SHAPE_DISK: return kPi * s.r * s.r;
    case SHAPE_CUBE: return 24.f;
    case SHAPE_CYLINDER: return kTwoPi * s.r * (s.z1 - s.z0);
    default: return 0.f;
  }
}

// Shape::point_pivot_pdf (shape.cpp:15-26): solid-angle pdf, in shape space,
// of sampling direction w (unit) from pivot by area sampling.
DG_HD float shape_generic_pivot_pdf(const DevShape& s, V3 pivot, V3 w) {
  float t;
  uint32_t face;
  if(!shape_hit<false>(s, pivot, w, 0.f, INFINITY, t, face)) { return 0.f; }
  V3 pt = madd_rn(pivot, w, t);
  V3 n = shape_local_normal(s, pt, face);
  return (1.f / shape_area(s)) * length_sq(pt - pivot) / fabsf(dot(w, n));
}

// point_pivot_pdf of the light shapes (sphere: sphere_shape.cpp:111-121).
DG_HD float shape_pivot_pdf(const DevShape& s, V3 pivot, V3 w) {
  if(s.kind == SHAPE_SPHERE) {
    float d2 = length_sq(pivot), r2 = s.r * s.r;
    if(d2 - r2 < 1e-3f) { return shape_generic_pivot_pdf(s, pivot, w); }
    float dist = sqrtf(d2);
    return uniform_cone_pdf(sqrtf(d2 - r2) / dist);
  }
  return shape_generic_pivot_pdf(s, pivot, w);
}

// sample_point_pivot of the light shapes, in shape space: the sampled point,
// its normal, the solid-angle pdf and the point's ray epsilon.
//   sphere: sphere_shape.cpp:74-109 (cone of directions towards the sphere
//           from outside; from inside, the reference's uniform-sphere branch
//           with its own pdf arithmetic, restated as it is)
//   disk:   Shape::sample_point_pivot (shape.cpp:4-13) over
//           DiskShape::sample_point (disk_shape.cpp:66-73)
DG_HD V3 shape_sample_pivot(const DevShape& s, V3 pivot, float u, float v, V3& n,
                            float& dir_pdf, float& eps) {
  if(s.kind == SHAPE_SPHERE) {
    float d2 = length_sq(pivot), r2 = s.r * s.r;
    eps = 5e-3f * s.r;
    if(d2 - r2 < 1e-3f) {
      V3 w = uniform_sphere_sample(u, v);
      V3 pt = w * s.r;
      float area_pdf = kInvFourPi / shape_area(s);
      dir_pdf = area_pdf * fabsf(dot(normalize(pivot - pt), w)) / length_sq(pivot - pt);
      n = w;
      return pt;
    }
    float dist = sqrtf(d2);
    float inv_dist = 1.f / dist;
    float cos_max = sqrtf(d2 - r2) * inv_dist;
    V3 cv = uniform_cone_sample(cos_max, u, v);
    V3 cz = -pivot * inv_dist;
    V3 cx, cy;
    coordinate_system(cz, cx, cy);
    V3 dir = cx * cv.x + cy * cv.y + cz * cv.z;
    float t;
    uint32_t face;
    if(!shape_hit<false>(s, pivot, dir, 0.f, INFINITY, t, face)) { t = dist; }
    V3 pt = madd_rn(pivot, dir, t);
    n = pt * (1.f / s.r);
    dir_pdf = uniform_cone_pdf(cos_max);
    return pt;
  }
  // disk (the only other light shape)
  float dx, dy;
  uniform_disk_sample(u, v, dx, dy);
  V3 pt = v3(dx * s.r, dy * s.r, s.z0);
  n = v3(0.f, 0.f, 1.f);
  eps = 1e-3f;
  float pos_pdf = kInvPi / (s.r * s.r);
  dir_pdf = pos_pdf * length_sq(pivot - pt) / fabsf(dot(n, normalize(pivot - pt)));
  return pt;
}

}  // namespace dort_gpu
