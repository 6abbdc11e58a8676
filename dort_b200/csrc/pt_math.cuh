// Vector arithmetic and the Monte Carlo sampling routines of the path
// tracer (src/dort/monte_carlo.cpp, geometry.cpp), for the device and the
// host.
#pragma once
#include <cmath>

#include "trace.cuh"

namespace dort_gpu {

// sin(pi x) and cos(pi x).  Every angle the samplers draw is 2 pi u or pi u
// for u in [0, 1), and sincospif needs no large-argument reduction for it.
#ifdef __CUDA_ARCH__
#define DG_SINCOSPI(x, s, c) sincospif((x), &(s), &(c))
#else
#define DG_SINCOSPI(x, s, c) \
  do { (s) = sinf(3.14159265358979323846f * (x)); (c) = cosf(3.14159265358979323846f * (x)); } while(0)
#endif
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
  float sn, cs;
  DG_SINCOSPI(2.f * u2, sn, cs);   // theta = 2 pi u2
  float x = cs * r, y = sn * r;
  float z = sqrtf(fmaxf(0.f, 1.f - x * x - y * y));
  return v3(x, y, z);
}
DG_HD float cosine_hemisphere_pdf(float cos_theta) { return fabsf(cos_theta * kInvPi); }
DG_HD V3 uniform_sphere_sample(float u1, float u2) {
  float z = 1.f - 2.f * u1;
  float r = sqrtf(fmaxf(0.f, 1.f - z * z));
  float sn, cs;
  DG_SINCOSPI(2.f * u2, sn, cs);   // phi = 2 pi u2
  return v3(cs * r, sn * r, z);
}
DG_HD V3 power_cosine_hemisphere_sample(float u1, float u2, float e) {
  float ct = powf(u2, 1.f / (1.f + e));
  float st = sqrtf(1.f - ct * ct);
  float sn, cs;
  DG_SINCOSPI(2.f * u1, sn, cs);   // phi = 2 pi u1
  return v3(cs * st, sn * st, ct);
}
DG_HD float power_cosine_hemisphere_pdf(float ct, float e) {
  return (e + 1.f) * powf(ct, e) * kInvTwoPi;
}

// monte_carlo.cpp:32-36
DG_HD void uniform_disk_sample(float u1, float u2, float& x, float& y) {
  float r = sqrtf(u1);
  float sn, cs;
  DG_SINCOSPI(2.f * u2, sn, cs);   // theta = 2 pi u2
  x = cs * r;
  y = sn * r;
}
// monte_carlo.cpp:56-68 (lerp(u1, 1, cos_max) = (1 - u1) + u1 cos_max)
DG_HD V3 uniform_cone_sample(float cos_max, float u1, float u2) {
  float ct = (1.f - u1) + u1 * cos_max;
  float st = sqrtf(fmaxf(0.f, 1.f - ct * ct));
  float sn, cs;
  DG_SINCOSPI(2.f * u2, sn, cs);   // phi = 2 pi u2
  return v3(cs * st, sn * st, ct);
}
DG_HD float uniform_cone_pdf(float cos_max) { return 1.f / (kTwoPi * (1.f - cos_max)); }

}  // namespace dort_gpu
