// Whole-scene harness around the reference renderer's "pt" and "lt" renderers.
//
// TEST INFRASTRUCTURE ONLY: compiled with the reference's sources by
// oracle/Makefile into oracle/_ref/.  Renders a scene given in the product's
// own C-ABI description (dort_scene_desc + dort_render_params of
// include/dort_gpu.h) with the reference's current code, so that the parity
// tests can tell a difference of the GPU path from a difference of the
// reference's stored test images.  Nothing in the product links it.
//
// The scene is assembled as the reference's builder assembles it
// (src/dort/lua_builder.cpp):
//   - plain triangles: TriangleShapePrimitive (lua_builder.cpp:375-390);
//   - emissive triangles: ShapePrimitive(TriangleShape) + DiffuseLight;
//   - analytic shapes: ShapePrimitive(SphereShape / DiskShape / CubeShape /
//     CylinderShape, transform) (lua_builder.cpp:327-348), emissive ones with
//     a DiffuseLight under the light's own transform (lua_light.cpp:87-97);
//   - PointLight / DirectionalLight (lua_light.cpp:45-74), InfiniteLight,
//     EnvironmentLight;
//   - the frame as lua_make_aggregate would (BvhPrimitive, middle split),
//     bounds / centroid / radius / background lights as build_scene;
//   - PinholeCamera / OrthoCamera / ThinLensCamera from the camera columns;
//   - PathRenderer (or LightRenderer for renderer = lt, path lengths = depths
//     + 2; BdptRenderer for renderer = bdpt, no debug images) with the render
//     parameters, RandomSampler(1, seed)
//     split(seed), box filter of radius 0.5 (lua_render.cpp:102-145).
#include <chrono>
#include <cmath>
#include <memory>
#include <vector>

#include "dort/bdpt_renderer.hpp"
#include "dort/bvh_primitive.hpp"
#include "dort/ctx.hpp"
#include "dort/cube_shape.hpp"
#include "dort/cylinder_shape.hpp"
#include "dort/dielectric_material.hpp"
#include "dort/diffuse_light.hpp"
#include "dort/directional_light.hpp"
#include "dort/disk_shape.hpp"
#include "dort/environment_light.hpp"
#include "dort/film.hpp"
#include "dort/filter.hpp"
#include "dort/image.hpp"
#include "dort/infinite_light.hpp"
#include "dort/lambert_material.hpp"
#include "dort/list_primitive.hpp"
#include "dort/mesh.hpp"
#include "dort/mirror_material.hpp"
#include "dort/oren_nayar_material.hpp"
#include "dort/ortho_camera.hpp"
#include "dort/light_renderer.hpp"
#include "dort/path_renderer.hpp"
#include "dort/phong_material.hpp"
#include "dort/pinhole_camera.hpp"
#include "dort/point_light.hpp"
#include "dort/primitive.hpp"
#include "dort/random_sampler.hpp"
#include "dort/rng.hpp"
#include "dort/scene.hpp"
#include "dort/sphere_shape.hpp"
#include "dort/texture.hpp"
#include "dort/thin_lens_camera.hpp"
#include "dort/thread_pool.hpp"
#include "dort/transform.hpp"
#include "dort/triangle_shape.hpp"
#include "dort/triangle_shape_primitive.hpp"

#include "dort_gpu.h"

namespace {
  using namespace dort;

  struct NoProgress final: public Progress {
    bool is_cancelled() const override { return false; }
    void set_percent_done(float) override { }
  };

  bool black(const float* c) { return c[0] == 0.f && c[1] == 0.f && c[2] == 0.f; }

  std::shared_ptr<Material> make_material(const dort_material& m) {
    Spectrum c(m.color[0], m.color[1], m.color[2]);
    Spectrum c2(m.color2[0], m.color2[1], m.color2[2]);
    switch(m.kind) {
      case DORT_MAT_MIRROR:
        return std::make_shared<MirrorMaterial>(const_texture<Spectrum>(c));
      case DORT_MAT_DIELECTRIC:
        return std::make_shared<DielectricMaterial>(const_texture<Spectrum>(c),
            const_texture<Spectrum>(c2), m.param[0] != 0.f ? m.param[0] : 1.5f,
            m.param[1] != 0.f ? m.param[1] : 1.f, m.param[2] != 0.f);
      case DORT_MAT_PHONG:
        return std::make_shared<PhongMaterial>(const_texture<Spectrum>(c),
            const_texture<Spectrum>(c2), const_texture<float>(m.param[0]));
      case DORT_MAT_CONDUCTOR:
        // no GGX conductor in the reference; a Phong stand-in for timing
        return std::make_shared<PhongMaterial>(const_texture<Spectrum>(Spectrum(0.f)),
            const_texture<Spectrum>(c),
            const_texture<float>(2.f / (m.param[0] * m.param[0]) - 2.f));
      case DORT_MAT_OREN_NAYAR:
        return std::make_shared<OrenNayarMaterial>(const_texture<Spectrum>(c),
            const_texture<float>(m.param[0]));
      default:
        return std::make_shared<LambertMaterial>(const_texture<Spectrum>(c));
    }
  }

  // Affine 3x4 row-major transform and its inverse as a reference Transform.
  Transform make_transform(const float* r) {
    Mat4x4 m(1.f), mi(1.f);
    for(int row = 0; row < 3; ++row) {
      for(int col = 0; col < 4; ++col) { m.cols[col][row] = r[4 * row + col]; }
    }
    double a = r[0], b = r[1], c = r[2], d = r[4], e = r[5], f = r[6], g = r[8], h = r[9],
           i = r[10];
    double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    double det = a * A + b * B + c * C;
    double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                     B / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                     C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
    for(int row = 0; row < 3; ++row) {
      double t = 0.0;
      for(int col = 0; col < 3; ++col) {
        mi.cols[col][row] = float(inv[3 * row + col]);
        t += inv[3 * row + col] * r[4 * col + 3];
      }
      mi.cols[3][row] = float(-t);
    }
    return Transform(m, mi);
  }

  std::shared_ptr<Shape> make_shape(const dort_shape& s) {
    switch(s.kind) {
      case DORT_SHAPE_SPHERE: return std::make_shared<SphereShape>(s.param[0]);
      case DORT_SHAPE_DISK: return std::make_shared<DiskShape>(s.param[0], s.param[1]);
      case DORT_SHAPE_CUBE: return std::make_shared<CubeShape>();
      default: return std::make_shared<CylinderShape>(s.param[0], s.param[1], s.param[2]);
    }
  }
}

extern "C" int dref_scene_render(const dort_scene_desc* d, const dort_render_params* rp,
                                 float* out_rgb, double* out_seconds) {
  auto pool = std::make_shared<ThreadPool>();
  pool->start(1);
  auto mesh = std::make_shared<Mesh>();
  for(uint32_t i = 0; i < d->vert_count; ++i) {
    mesh->points.push_back(Point(d->verts[3 * i], d->verts[3 * i + 1], d->verts[3 * i + 2]));
  }
  mesh->vertices.assign(d->tris, d->tris + 3 * size_t(d->tri_count));

  std::vector<std::shared_ptr<Material>> materials;
  for(uint32_t i = 0; i < d->material_count; ++i) {
    materials.push_back(make_material(d->materials[i]));
  }
  if(materials.empty()) {
    materials.push_back(std::make_shared<LambertMaterial>(const_texture<Spectrum>(Spectrum(0.5f))));
  }

  // the triangles lights sample when they differ from their primitives
  auto light_mesh = std::make_shared<Mesh>();
  std::vector<std::unique_ptr<Primitive>> prims;
  std::vector<std::shared_ptr<Light>> lights;
  for(uint32_t t = 0; t < d->tri_count; ++t) {
    auto mat = materials.at(d->tri_material ? d->tri_material[t] : 0);
    const float* le = d->tri_emission ? d->tri_emission + 3 * size_t(t) : nullptr;
    if(le && !black(le)) {
      auto shape = std::make_shared<TriangleShape>(mesh.get(), 3 * t);
      std::shared_ptr<Shape> light_shape = shape;
      if(d->tri_light_verts) {
        const float* lv = d->tri_light_verts + 9 * size_t(t);
        uint32_t base = uint32_t(light_mesh->points.size());
        for(int k = 0; k < 3; ++k) {
          light_mesh->points.push_back(Point(lv[3 * k], lv[3 * k + 1], lv[3 * k + 2]));
          light_mesh->vertices.push_back(base + uint32_t(k));
        }
        light_shape = std::make_shared<TriangleShape>(light_mesh.get(), base);
      }
      auto light = std::make_shared<DiffuseLight>(light_shape, identity(),
          Spectrum(le[0], le[1], le[2]));
      prims.push_back(std::make_unique<ShapePrimitive>(shape, mat, light, identity()));
      lights.push_back(light);
    } else {
      prims.push_back(std::make_unique<TriangleShapePrimitive>(mesh.get(), 3 * t, mat));
    }
  }
  for(uint32_t k = 0; k < d->shape_count; ++k) {
    const dort_shape& s = d->shapes[k];
    auto shape = make_shape(s);
    Transform t = make_transform(s.to_world);
    std::shared_ptr<Light> light;
    if(!black(s.emission)) {
      Transform lt = (s.flags & DORT_SHAPE_LIGHT_TRANSFORM) ? make_transform(s.light_to_world) : t;
      light = std::make_shared<DiffuseLight>(shape, lt,
          Spectrum(s.emission[0], s.emission[1], s.emission[2]));
      lights.push_back(light);
    }
    prims.push_back(std::make_unique<ShapePrimitive>(shape, materials.at(s.material), light, t));
  }
  for(uint32_t k = 0; k < d->light_count; ++k) {
    const dort_light& l = d->lights[k];
    Spectrum c(l.rgb[0], l.rgb[1], l.rgb[2]);
    if(l.kind == DORT_LIGHT_POINT) {
      lights.push_back(std::make_shared<PointLight>(Point(l.vec[0], l.vec[1], l.vec[2]), c));
    } else {
      lights.push_back(std::make_shared<DirectionalLight>(Vector(l.vec[0], l.vec[1], l.vec[2]), c));
    }
  }

  BvhOpts opts;
  auto scene = std::make_shared<Scene>();
  if(prims.size() == 1) {
    scene->primitive = std::move(prims.at(0));
  } else if(prims.size() <= opts.leaf_size) {
    scene->primitive = std::make_unique<ListPrimitive>(std::move(prims));
  } else {
    scene->primitive = std::make_unique<BvhPrimitive>(std::move(prims), opts, *pool);
  }
  scene->bounds = scene->primitive->bounds();
  scene->centroid = scene->bounds.centroid();
  scene->radius = scene->bounds.radius();
  if(!black(d->sky_const)) {
    lights.push_back(std::make_shared<InfiniteLight>(
          Spectrum(d->sky_const[0], d->sky_const[1], d->sky_const[2])));
  }
  if(d->sky_rgb && d->sky_width > 0 && d->sky_height > 0) {
    auto img = std::make_shared<Image<PixelRgbFloat>>(d->sky_width, d->sky_height);
    for(uint32_t y = 0; y < d->sky_height; ++y) {
      for(uint32_t x = 0; x < d->sky_width; ++x) {
        const float* p = d->sky_rgb + 3 * (size_t(y) * d->sky_width + x);
        img->set_rgb(x, y, Spectrum(p[0], p[1], p[2]));
      }
    }
    Spectrum sc = black(d->sky_scale) ? Spectrum(1.f)
      : Spectrum(d->sky_scale[0], d->sky_scale[1], d->sky_scale[2]);
    Vector up = black(d->sky_up) ? Vector(0.f, 1.f, 0.f)
      : Vector(d->sky_up[0], d->sky_up[1], d->sky_up[2]);
    Vector fwd = black(d->sky_fwd) ? Vector(1.f, 0.f, 0.f)
      : Vector(d->sky_fwd[0], d->sky_fwd[1], d->sky_fwd[2]);
    lights.push_back(std::make_shared<EnvironmentLight>(img, sc, up, fwd));
  }
  scene->lights = lights;
  for(const auto& light: scene->lights) {
    if(light->flags & LIGHT_BACKGROUND) { scene->background_lights.push_back(light); }
  }
  scene->meshes.push_back(mesh);
  scene->meshes.push_back(light_mesh);

  const dort_camera& c = rp->camera;
  Mat4x4 m(1.f);
  for(int r = 0; r < 3; ++r) {
    m.cols[0][r] = c.right[r];
    m.cols[1][r] = c.up[r];
    m.cols[2][r] = c.forward[r];
    m.cols[3][r] = c.origin[r];
  }
  float rows[12];
  for(int r = 0; r < 3; ++r) {
    for(int col = 0; col < 4; ++col) { rows[4 * r + col] = m.cols[col][r]; }
  }
  Transform cam_t = make_transform(rows);
  std::shared_ptr<Camera> camera;
  if(c.kind == DORT_CAMERA_ORTHO) {
    camera = std::make_shared<OrthoCamera>(cam_t, c.dimension);
  } else if(c.kind == DORT_CAMERA_THIN_LENS) {
    camera = std::make_shared<ThinLensCamera>(cam_t, c.fov, c.lens_radius, c.focal_distance);
  } else {
    float fov = c.fov < 1e-2f ? 1e-2f : (c.fov > PI ? PI : c.fov);
    camera = std::make_shared<PinholeCamera>(cam_t, fov);
  }

  auto film = std::make_shared<Film>(rp->width, rp->height,
      std::make_shared<BoxFilter>(Vec2(0.5f, 0.5f)));
  uint32_t seed = uint32_t(rp->seed);
  std::shared_ptr<Sampler> sampler =
    std::make_shared<RandomSampler>(1, Rng(seed))->split(seed);
  PathRenderer::DirectStrategy ds = rp->direct_strategy == 1
    ? PathRenderer::DirectStrategy::SAMPLE_BSDF
    : rp->direct_strategy == 2 ? PathRenderer::DirectStrategy::SAMPLE_LIGHT
    : PathRenderer::DirectStrategy::MIS;
  std::unique_ptr<Renderer> renderer;
  if(rp->renderer == DORT_RENDERER_LT) {
    // dort.render.make for "lt": path lengths = depths + 2 (lua_render.cpp:146-150)
    renderer.reset(new LightRenderer(scene, film, sampler, camera, rp->iterations,
        rp->min_depth + 2, rp->max_depth + 2));
  } else if(rp->renderer == DORT_RENDERER_BDPT) {
    // dort.render.make for "bdpt" (lua_render.cpp:151-159)
    renderer.reset(new BdptRenderer(scene, film, sampler, camera, rp->iterations,
        rp->min_depth, rp->max_depth, (rp->renderer_flags & DORT_BDPT_NO_T1_PATHS) == 0, ""));
  } else {
    renderer.reset(new PathRenderer(scene, film, sampler, camera, rp->iterations,
        rp->min_depth, rp->max_depth, rp->only_direct != 0, rp->sample_all_lights != 0, ds));
  }
  CtxG ctx;
  ctx.pool = pool;
  NoProgress progress;
  auto t0 = std::chrono::steady_clock::now();
  renderer->render(ctx, progress);
  auto t1 = std::chrono::steady_clock::now();
  if(out_seconds) { *out_seconds = std::chrono::duration<double>(t1 - t0).count(); }
  Image<PixelRgbFloat> img = film->to_image<PixelRgbFloat>();
  for(uint32_t y = 0; y < rp->height; ++y) {
    for(uint32_t x = 0; x < rp->width; ++x) {
      PixelRgbFloat p = img.get_pixel(x, y);
      float* o = out_rgb + 3 * (size_t(y) * rp->width + x);
      o[0] = p.r; o[1] = p.g; o[2] = p.b;
    }
  }
  pool->stop();
  return 0;
}
