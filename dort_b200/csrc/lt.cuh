// Light tracing: the "lt" renderer (LightRenderer, light_renderer.cpp:13-181).
//
// Every path starts on a light picked in proportion to its power: its first
// vertex is connected straight to the camera (sample_immediate, :108-147),
// then the path is traced from the light with the adjoint BSDF sampling
// (Bsdf::sample_camera_f) and every non-delta vertex is connected to the
// camera (connect_to_camera, :149-180); contributions are splatted onto the
// film (Film::add_splat, film.cpp:32-67; the box filter of radius 1/2 puts a
// splat on the pixel that contains its film position) and the film is
// scaled by 1 / iterations (:42).  W x H x iterations paths per frame.
//
// Light emission (Light::sample_ray_radiance / sample_point / eval_radiance)
// and camera importance (Camera::sample_pivot_importance / sample_point /
// eval_importance) are restated for every light and camera kind the path
// tracer supports.
#pragma once
#include "pt.cuh"

namespace dort_gpu {

// ---- camera importance ----------------------------------------------------------------

// World -> camera coordinates (Transform::apply_inv of the camera transform).
DG_HD V3 cam_local_vec(const PtParams& pp, V3 w) {
  return v3(pp.cam_inv[0] * w.x + pp.cam_inv[1] * w.y + pp.cam_inv[2] * w.z,
            pp.cam_inv[3] * w.x + pp.cam_inv[4] * w.y + pp.cam_inv[5] * w.z,
            pp.cam_inv[6] * w.x + pp.cam_inv[7] * w.y + pp.cam_inv[8] * w.z);
}
DG_HD V3 cam_local_point(const PtParams& pp, V3 p) { return cam_local_vec(pp, p - v3p(pp.origin)); }
DG_HD V3 cam_world_point(const PtParams& pp, V3 c) {
  return v3p(pp.origin) + v3p(pp.right) * c.x + v3p(pp.up) * c.y + v3p(pp.forward) * c.z;
}

// get_image_plane_area of the pinhole / thin lens (pinhole_camera.cpp:124-127,
// thin_lens_camera.cpp:116-119) and the orthographic camera (ortho_camera.cpp:90-93).
DG_HD float image_plane_area(const PtParams& pp) {
  float w = float(pp.width), h = float(pp.height);
  float aspect = fminf(w, h) / fmaxf(w, h);
  if(pp.camera == CAMERA_ORTHO) { return sq(pp.ortho_dim) * aspect; }
  return aspect * sq(pp.proj_dim);
}

// Film position of a direction on the image plane z = 1 given as the plane
// position (px, py) (the common tail of the pinhole and thin-lens
// get_film_pos, pinhole_camera.cpp:107-122).
DG_HD bool plane_film_pos(const PtParams& pp, float px, float py, float& fx, float& fy) {
  float nx = px / pp.proj_dim, ny = py / pp.proj_dim;
  if(fabsf(nx) > 0.5f || fabsf(ny) > 0.5f) { return false; }
  float w = float(pp.width), h = float(pp.height);
  float cx = w > h ? nx : nx * h / w;
  float cy = w > h ? ny * w / h : ny;
  fx = (cx + 0.5f) * w;
  fy = (cy + 0.5f) * h;
  return true;
}

// ThinLensCamera::get_film_pos (thin_lens_camera.cpp:121-139).
DG_HD bool thin_film_pos(const PtParams& pp, V3 lens, V3 pivot, float& fx, float& fy) {
  if(pivot.z <= 0.f) { return false; }
  float t = pp.focal_distance / pivot.z;
  V3 fp = lens + (pivot - lens) * t;
  return plane_film_pos(pp, fp.x / fp.z, fp.y / fp.z, fx, fy);
}

// OrthoCamera::get_film_pos (ortho_camera.cpp:72-82).
DG_HD bool ortho_film_pos(const PtParams& pp, V3 c, float& fx, float& fy) {
  if(c.z < 0.f) { return false; }
  float w = float(pp.width), h = float(pp.height);
  float fd = fmaxf(w, h);
  fx = (c.x / pp.ortho_dim + 0.5f) * fd;
  fy = (c.y / pp.ortho_dim + 0.5f) * fd;
  return fx >= 0.f && fx <= w && fy >= 0.f && fy <= h;
}

struct CameraPivot {
  V3 p;             // point on the camera
  float fx, fy;     // film position
  float pdf;        // area pdf of p given the pivot
  float We;         // importance
};

// Camera::sample_pivot_importance (pinhole_camera.cpp:34-56,
// thin_lens_camera.cpp:35-53, ortho_camera.cpp:28-46); false = no importance.
template<bool G>
DG_HD bool camera_pivot_importance(const PtParams& pp, V3 pivot, float u, float v,
                                   CameraPivot& out) {
  V3 c = cam_local_point(pp, pivot);
  float area = image_plane_area(pp);
  if(G && pp.camera == CAMERA_THIN_LENS) {
    float lx, ly;
    uniform_disk_sample(u, v, lx, ly);
    V3 lens = v3(lx * pp.lens_radius, ly * pp.lens_radius, 0.f);
    if(!thin_film_pos(pp, lens, c, out.fx, out.fy)) { return false; }
    out.p = cam_world_point(pp, lens);
    out.pdf = kInvPi / sq(pp.lens_radius);
    out.We = kInvPi / (sq(pp.lens_radius) * area);
    return true;
  }
  if(G && pp.camera == CAMERA_ORTHO) {
    if(!ortho_film_pos(pp, c, out.fx, out.fy)) { return false; }
    float w = float(pp.width), h = float(pp.height);
    float k = pp.ortho_dim / fmaxf(w, h);
    V3 plane = v3((out.fx - 0.5f * w) * k, (out.fy - 0.5f * h) * k, 0.f);
    out.p = cam_world_point(pp, plane);
    out.pdf = 1.f / length_sq(out.p - pivot);
    out.We = 1.f / area;
    return true;
  }
  if(c.z <= 0.f) { return false; }
  if(!plane_film_pos(pp, c.x / c.z, c.y / c.z, out.fx, out.fy)) { return false; }
  float cos_t = c.z / length(c);
  out.p = v3p(pp.origin);
  out.pdf = 1.f;
  out.We = 1.f / (area * cos_t * cos_t * cos_t);
  return true;
}

// Camera::sample_point (pinhole_camera.cpp:58-61, thin_lens_camera.cpp:55-61,
// ortho_camera.cpp:48-55).
template<bool G>
DG_HD V3 camera_sample_point(const PtParams& pp, float u, float v, float& pdf) {
  if(G && pp.camera == CAMERA_THIN_LENS) {
    float lx, ly;
    uniform_disk_sample(u, v, lx, ly);
    pdf = kInvPi / sq(pp.lens_radius);
    return cam_world_point(pp, v3(lx * pp.lens_radius, ly * pp.lens_radius, 0.f));
  }
  if(G && pp.camera == CAMERA_ORTHO) {
    float w = float(pp.width), h = float(pp.height);
    float k = pp.ortho_dim / fmaxf(w, h);
    float fx = u * w, fy = v * h;
    pdf = 1.f / image_plane_area(pp);
    return cam_world_point(pp, v3((fx - 0.5f * w) * k, (fy - 0.5f * h) * k, 0.f));
  }
  pdf = 1.f;
  return v3p(pp.origin);
}

// Camera::eval_importance from a camera point p towards wi
// (pinhole_camera.cpp:63-82, thin_lens_camera.cpp:63-77; the orthographic
// camera has none, ortho_camera.cpp:57-59).
template<bool G>
DG_HD float camera_eval_importance(const PtParams& pp, V3 p, V3 wi, float& fx, float& fy) {
  float area = image_plane_area(pp);
  if(G && pp.camera == CAMERA_ORTHO) { return 0.f; }
  if(G && pp.camera == CAMERA_THIN_LENS) {
    V3 lens = cam_local_point(pp, p);
    V3 dir = cam_local_vec(pp, wi);
    if(!thin_film_pos(pp, lens, dir + lens, fx, fy)) { return 0.f; }
    float cos_t = dir.z / length(dir);
    return kInvPi / (sq(pp.lens_radius) * area * cos_t * cos_t * cos_t);
  }
  V3 c = cam_local_vec(pp, wi);
  if(c.z <= 0.f) { return 0.f; }
  if(!plane_film_pos(pp, c.x / c.z, c.y / c.z, fx, fy)) { return 0.f; }
  float cos_t = c.z / length(c);
  return 1.f / (area * cos_t * cos_t * cos_t);
}

// ---- light emission ---------------------------------------------------------------------

// uniform_hemisphere_sample (monte_carlo.cpp:6-13)
DG_HD V3 uniform_hemisphere_sample(float u1, float u2) {
  float z = u1;
  float r = sqrtf(fmaxf(0.f, 1.f - z * z));
  float s, c;
  DG_SINCOSPI(2.f * u2, s, c);
  return v3(c * r, s * r, z);
}

struct LightPoint {
  V3 p, nn;         // point and unit normal (zero for a point light)
  float eps;        // ray epsilon at p
  float pos_pdf;    // area pdf
};

// Light::sample_point: triangles (triangle.cpp:62-76), spheres and disks
// (sphere_shape.cpp:62-70, disk_shape.cpp:65-73) through DiffuseLight
// (diffuse_light.cpp:70-83), point lights (point_light.cpp:33-41); distant
// lights have no point (false).
template<bool G>
DG_HD bool light_sample_point(const PtScene& sc, const DevLight& l, float u, float v,
                              LightPoint& out) {
  if(l.kind == LIGHT_TRI) {
    float s = sqrtf(u);
    float b1 = 1.f - s, b2 = v * s;
    out.p = v3p(l.p0) + b1 * v3p(l.e1) + b2 * v3p(l.e2);
    out.nn = v3p(l.nn);
    out.eps = 1e-3f;
    out.pos_pdf = 1.f / l.area;
    return true;
  }
  if(G && l.kind == LIGHT_SHAPE) {
    const DevShape& sh = sc.light_shapes[l.tri];
    V3 pl, nl;
    if(sh.kind == SHAPE_SPHERE) {
      V3 w = uniform_sphere_sample(u, v);
      pl = w * sh.r;
      nl = w;
      out.eps = 5e-3f * sh.r;
    } else {
      float x, y;
      uniform_disk_sample(u, v, x, y);
      pl = v3(x * sh.r, y * sh.r, sh.z0);
      nl = v3(0.f, 0.f, 1.f);
      out.eps = 1e-3f;
    }
    out.p = xf_point(sh.m, pl);
    out.nn = normalize(xf_normal(sh.inv, nl));
    out.pos_pdf = 1.f / l.area;
    return true;
  }
  if(G && l.kind == LIGHT_POINT) {
    out.p = v3p(l.p0);
    out.nn = v3(0.f, 0.f, 0.f);
    out.eps = 0.f;
    out.pos_pdf = 1.f;
    return true;
  }
  return false;
}

// Light::eval_radiance from a sampled light point towards a pivot
// (diffuse_light.cpp:85-94 one-sided; point_light.cpp:43-47).
template<bool G>
DG_HD V3 light_eval_radiance(const PtScene& sc, const DevLight& l, V3 p, V3 nn, V3 pivot) {
  if(G && l.kind == LIGHT_POINT) { return v3p(l.L) * (1.f / length_sq(v3p(l.p0) - pivot)); }
  if(light_is_area(l)) { return area_eval_radiance(sc, l, p, nn, pivot); }
  return v3(0.f, 0.f, 0.f);
}

struct LightRay {
  V3 o, d;          // origin and unit direction
  V3 nn;            // normal at the origin (the direction for point and distant lights)
  V3 L;             // radiance / intensity
  float eps;        // ray epsilon
  float pos_pdf, dir_pdf;
};

// Light::sample_ray_radiance for every light kind: area lights
// (diffuse_light.cpp:15-38: a uniform hemisphere direction on the side of the
// normal, pdf 1 / 2 pi), point lights (point_light.cpp:6-17), directional
// lights (directional_light.cpp:13-26), the constant sky (infinite_light.cpp:
// 5-23) and the environment map (environment_light.cpp:34-53); distant lights
// start on a disk of the scene's bounding sphere.
template<bool G>
DG_HD bool light_sample_ray(const PtScene& sc, const DevLight& l, float u1, float u2, float u3,
                            float u4, LightRay& out) {
  if(light_is_area(l)) {
    LightPoint lp;
    if(!light_sample_point<G>(sc, l, u1, u2, lp)) { return false; }
    // a uniform direction folded onto the normal's side: uniform over that
    // hemisphere whatever the frame (the reference folds in shape space and
    // carries the direction to the world; the same distribution for the
    // rigid light transforms of the scenes here)
    V3 w = uniform_hemisphere_sample(u3, u4);
    if(dot(w, lp.nn) < 0.f) { w = -w; }
    out.o = lp.p;
    out.d = w;
    out.nn = lp.nn;
    out.L = light_radiance(sc, l);
    out.eps = lp.eps;
    out.pos_pdf = lp.pos_pdf;
    out.dir_pdf = kInvTwoPi;
    return true;
  }
  if(G && l.kind == LIGHT_POINT) {
    V3 w = uniform_sphere_sample(u3, u4);
    out.o = v3p(l.p0);
    out.d = w;
    out.nn = w;
    out.L = v3p(l.L);
    out.eps = 0.f;
    out.pos_pdf = 1.f;
    out.dir_pdf = kInvFourPi;
    return true;
  }
  V3 c = v3p(sc.centroid);
  float r = sc.radius;
  float dx, dy;
  uniform_disk_sample(u1, u2, dx, dy);
  out.eps = 0.f;
  out.pos_pdf = kInvPi / sq(r);
  if(G && l.kind == LIGHT_DIR) {
    V3 dir = v3p(l.nn), s, t;
    coordinate_system(dir, s, t);
    out.o = c + r * (-dir + dx * s + dy * t);
    out.d = dir;
    out.nn = dir;
    out.L = v3p(l.L);
    out.dir_pdf = 1.f;
    return true;
  }
  if(l.kind == LIGHT_INFINITE) {
    V3 dir = uniform_sphere_sample(u3, u4), s, t;
    coordinate_system(dir, s, t);
    out.o = c + r * (-dir + dx * s + dy * t);
    out.d = dir;
    out.nn = dir;
    out.L = v3p(l.L);
    out.dir_pdf = kInvFourPi;
    return true;
  }
  if(l.kind == LIGHT_ENV) {
    float du, dv, pdf;
    V3 dir = env_sample_dir(sc.env, u3, u4, du, dv, pdf), s, t;
    coordinate_system(dir, s, t);
    out.o = c + r * (dir + dx * s + dy * t);
    out.d = -dir;
    out.nn = -dir;
    out.L = env_radiance_uv(sc.env, du, dv);
    out.dir_pdf = pdf;
    return true;
  }
  return false;
}

// ---- the light path -------------------------------------------------------------

// Dimension blocks of one light path:
//   0        light pick (a), light point uv (b, c), camera point u (d)
//   1        camera point v (a), ray position uv (b, c), ray direction u (d)
//   2        ray direction v (a)
//   3 + 2k   bounce k: camera point uv of the connection (a, b), BSDF uv (c, d)
//   4 + 2k   bounce k: BSDF component (a), roulette (b)
constexpr uint32_t kLtBounceBlock = 3;

// Film::add_splat with the box filter of radius 1/2: the pixel containing the
// film position (a position on a pixel edge falls to the pixel on its right
// or below; the reference splits it between both, an event of probability
// 0).  A position outside the film reaches no pixel's filter and is dropped:
// on films wider than high the pinhole's get_film_pos returns such positions
// (pinhole_camera.cpp:107-122 bounds the square [-1/2, 1/2]^2 before the
// aspect scaling), for which the reference's add_splat sizes its weight
// array from an empty pixel rectangle (film.cpp:32-41).
DG_HD void lt_splat(float* film, const PtParams& pp, float fx, float fy, V3 c) {
  if(!(c.x >= 0.f && c.y >= 0.f && c.z >= 0.f) || !isfinite(c.x + c.y + c.z)) { return; }
  if(!(fx >= 0.f && fx <= float(pp.width) && fy >= 0.f && fy <= float(pp.height))) { return; }
  int x = int(floorf(fx)), y = int(floorf(fy));
  x = x >= int(pp.width) ? int(pp.width) - 1 : x;
  y = y >= int(pp.height) ? int(pp.height) - 1 : y;
  float* px = film + 3 * (size_t(y) * pp.width + x);
#ifdef __CUDA_ARCH__
  atomicAdd(px, c.x);
  atomicAdd(px + 1, c.y);
  atomicAdd(px + 2, c.z);
#else
  px[0] += c.x;
  px[1] += c.y;
  px[2] += c.z;
#endif
}

// Unoccluded segment between two points (ShadowTest::init_point_point,
// light.cpp:40-49): from a with epsilon ea to b with epsilon eb.
template<bool G>
DG_HD bool lt_visible(const PtScene& sc, V3 a, float ea, V3 b, float eb) {
  V3 d = b - a;
  float dist = length(d);
  if(!(dist > 0.f)) { return false; }
  Hit h = scene_trace<true, G>(sc, a, ea, d * (1.f / dist), dist - eb);
  return h.prim == kMiss;
}

// One light path (LightRenderer::sample_path, light_renderer.cpp:49-105);
// returns the rays traced.
template<bool G>
DG_HD uint32_t lt_path(const PtScene& sc, const PtParams& pp, uint32_t pixel, uint32_t sample,
                       float* film) {
  uint32_t rays = 0;
  if(sc.light_count == 0) { return 0; }
  const uint32_t min_len = pp.min_depth + 2, max_len = pp.max_depth + 2;
  Rand4 r0 = rand4(pp.seed, pixel, sample, 0);
  Rand4 r1 = rand4(pp.seed, pixel, sample, 1);
  uint32_t li = distrib_sample(sc.light_cdf, sc.light_count + 1, r0.a);
  float pick = distrib_pdf(sc.light_cdf, sc.light_count + 1, li);
  if(pick == 0.f) { return 0; }
  const DevLight& l = sc.lights[li];

  // sample_immediate (light_renderer.cpp:108-147): light point straight to the camera
  if(min_len <= 2 && 2 <= max_len) {
    LightPoint lp;
    if(light_sample_point<G>(sc, l, r0.b, r0.c, lp) && lp.pos_pdf != 0.f) {
      float cam_pdf;
      V3 cp = camera_sample_point<G>(pp, r0.d, r1.a, cam_pdf);
      V3 to = lp.p - cp;
      if(cam_pdf != 0.f && !(to.x == 0.f && to.y == 0.f && to.z == 0.f)) {
        float fx, fy;
        float We = camera_eval_importance<G>(pp, cp, normalize(to), fx, fy);
        V3 Le = light_eval_radiance<G>(sc, l, lp.p, lp.nn, cp);
        float cpdf = pick * lp.pos_pdf * cam_pdf;
        if(We != 0.f && !is_black(Le) && cpdf != 0.f) {
          V3 c = Le * (We / (length_sq(to) * cpdf));
          if(!is_black(lp.nn)) { c = c * fabsf(dot(lp.nn, normalize(to))); }
          if(!is_black(c)) {
            ++rays;
            if(lt_visible<G>(sc, lp.p, lp.eps, cp, 0.f)) { lt_splat(film, pp, fx, fy, c); }
          }
        }
      }
    }
  }
  if(max_len < 3) { return rays; }

  Rand4 r2 = rand4(pp.seed, pixel, sample, 2);
  LightRay ray;
  if(!light_sample_ray<G>(sc, l, r1.b, r1.c, r1.d, r2.a, ray)) { return rays; }
  float light_pdf = pick * ray.pos_pdf * ray.dir_pdf;
  if(is_black(ray.L) || light_pdf == 0.f) { return rays; }
  V3 thr = ray.L * (1.f / (ray.pos_pdf * pick));
  float prev_dir_pdf = ray.dir_pdf;
  V3 prev_nn = ray.nn;
  V3 o = ray.o, d = ray.d;
  float eps = ray.eps;
  for(uint32_t b = 0; b + 3 <= max_len; ++b) {
    if(prev_dir_pdf == 0.f) { break; }
    ++rays;
    Hit h = scene_trace<false, G>(sc, o, eps, d, INFINITY);
    if(h.prim == kMiss) { break; }
    SurfaceHit g = surface_at<G>(sc, h, o, d);
    DevMaterial m = material_at(sc, g);
    V3 wi = -d;
    float geom = fabsf(dot(prev_nn, wi)) / prev_dir_pdf;
    Rand4 ra = rand4(pp.seed, pixel, sample, kLtBounceBlock + 2 * b);
    Rand4 rb = rand4(pp.seed, pixel, sample, kLtBounceBlock + 2 * b + 1);

    // connect_to_camera (light_renderer.cpp:149-180)
    if(b + 3 >= min_len && bxdf_matches(m.bxdf_flags, F_ALL & ~F_DELTA)) {
      CameraPivot cam;
      if(camera_pivot_importance<G>(pp, g.p, ra.a, ra.b, cam) && cam.pdf != 0.f && cam.We != 0.f) {
        V3 cw = cam.p - g.p;
        float dist2 = length_sq(cw);
        V3 cwo = normalize(cw);
        V3 f = bsdf_eval<G>(m, g.frame, wi, cwo, F_ALL);
        if(!is_black(f)) {
          V3 c = thr * geom * f * (cam.We * fabsf(dot(g.n, cwo)) / (dist2 * cam.pdf));
          if(!is_black(c)) {
            ++rays;
            if(lt_visible<G>(sc, g.p, g.eps, cam.p, 0.f)) { lt_splat(film, pp, cam.fx, cam.fy, c); }
          }
        }
      }
    }

    // Bsdf::sample_camera_f (bsdf.cpp:104-112): every BxDF here samples the
    // same way from either side (symmetric ones and the dielectric,
    // dielectric_material.cpp:17-22); shading_to_geom of the fixed direction
    BsdfSample s = bsdf_sample<G>(m, g.frame, wi, F_ALL, ra.c, ra.d, rb.a);
    if(s.pdf == 0.f) { break; }
    float dn = fabsf(dot(g.frame.n, wi));
    V3 contrib = (dn == 0.f) ? v3(0.f, 0.f, 0.f) : s.f * geom;
    thr = thr * contrib;
    if(is_black(thr)) { break; }
    if(b + 3 > min_len && b >= 2) {
      float survive = clampf(average(contrib), 0.1f, 0.9f);
      if(rb.b > survive) { break; }
      thr = thr * (1.f / survive);
    }
    prev_nn = g.n;
    prev_dir_pdf = s.pdf;
    o = g.p;
    d = normalize(s.w);
    eps = g.eps;
  }
  return rays;
}

}  // namespace dort_gpu
