// Path-tracing harness around the reference renderer's own "pt" renderer.
//
// TEST INFRASTRUCTURE ONLY: compiled with the reference's sources by
// oracle/Makefile into oracle/_ref/.  Produces converged reference images for
// the parity tests and is the CPU baseline ("reference" kind) for the render
// workloads.  Nothing in the product links it.
//
// The scene is assembled from a flat triangle description exactly the way the
// reference's Lua builder assembles a DSL scene (src/dort/lua_builder.cpp):
//   - a plain triangle is add_triangle -> TriangleShapePrimitive
//     (lua_builder.cpp:375-390);
//   - an emissive triangle is dort.builder.add_diffuse_light
//     (lua/dort/builder_ext.lua:38-48): a black Lambert material and a
//     ShapePrimitive(TriangleShape, DiffuseLight) plus add_light;
//   - the frame becomes one BvhPrimitive / ListPrimitive / primitive
//     (lua_make_aggregate, lua_builder.cpp:699-710) and build_scene fills the
//     bounds, centroid, radius and background lights (lua_builder.cpp:113-146);
//   - the renderer is PathRenderer with dort.render.make's parameters and
//     defaults (lua_render.cpp:102-145), sampler RandomSampler(1, seed)
//     split(seed), box filter of radius 0.5.
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "dort/bvh_primitive.hpp"
#include "dort/ctx.hpp"
#include "dort/dielectric_material.hpp"
#include "dort/diffuse_light.hpp"
#include "dort/environment_light.hpp"
#include "dort/film.hpp"
#include "dort/filter.hpp"
#include "dort/image.hpp"
#include "dort/infinite_light.hpp"
#include "dort/lambert_material.hpp"
#include "dort/list_primitive.hpp"
#include "dort/mesh.hpp"
#include "dort/mirror_material.hpp"
#include "dort/path_renderer.hpp"
#include "dort/phong_material.hpp"
#include "dort/pinhole_camera.hpp"
#include "dort/primitive.hpp"
#include "dort/random_sampler.hpp"
#include "dort/rng.hpp"
#include "dort/scene.hpp"
#include "dort/texture.hpp"
#include "dort/thread_pool.hpp"
#include "dort/transform.hpp"
#include "dort/triangle_shape.hpp"
#include "dort/triangle_shape_primitive.hpp"

namespace {
  using namespace dort;

  struct NoProgress final: public Progress {
    bool is_cancelled() const override { return false; }
    void set_percent_done(float) override { }
  };

  // Material record layout shared with the Python side: kind, color[3],
  // color2[3], param[4] (11 floats), kinds as in dort_gpu.h.
  std::shared_ptr<Material> make_material(const float* m) {
    uint32_t kind = uint32_t(m[0]);
    Spectrum c(m[1], m[2], m[3]);
    Spectrum c2(m[4], m[5], m[6]);
    switch(kind) {
      case 1:
        return std::make_shared<MirrorMaterial>(const_texture<Spectrum>(c));
      case 2:
        return std::make_shared<DielectricMaterial>(const_texture<Spectrum>(c),
            const_texture<Spectrum>(c2), m[7] > 0.f ? m[7] : 1.5f, 1.f, false);
      case 3:
        return std::make_shared<PhongMaterial>(const_texture<Spectrum>(c),
            const_texture<Spectrum>(c2), const_texture<float>(m[7]));
      case 4:
        // no GGX conductor in the reference; timed with a Phong stand-in
        return std::make_shared<PhongMaterial>(const_texture<Spectrum>(Spectrum(0.f)),
            const_texture<Spectrum>(c), const_texture<float>(2.f / (m[7] * m[7]) - 2.f));
      default:
        return std::make_shared<LambertMaterial>(const_texture<Spectrum>(c));
    }
  }

  std::shared_ptr<ThreadPool> pool_for(uint32_t threads) {
    static std::shared_ptr<ThreadPool> pool;
    static uint32_t started = 0;
    if(!pool || started != threads) {
      if(pool) { pool->stop(); }
      pool = std::make_shared<ThreadPool>();
      pool->start(threads);
      started = threads;
    }
    return pool;
  }
}

struct RefPtScene {
  std::shared_ptr<Scene> scene;
  std::shared_ptr<Mesh> mesh;
};

extern "C" void* dref_pt_scene_create(
    const float* verts, uint32_t vert_count, const uint32_t* tris, uint32_t tri_count,
    const uint32_t* tri_mat, const float* mats, uint32_t mat_count,
    const float* tri_emission,
    const float* bg_const, const float* env_rgb, uint32_t env_w, uint32_t env_h,
    const float* env_frame /* scale.rgb, up.xyz, fwd.xyz */,
    int split_method, uint32_t threads, double* out_build_s)
{
  auto pool = pool_for(threads);
  auto t0 = std::chrono::steady_clock::now();
  auto mesh = std::make_shared<Mesh>();
  for(uint32_t i = 0; i < vert_count; ++i) {
    mesh->points.push_back(Point(verts[3*i], verts[3*i + 1], verts[3*i + 2]));
  }
  mesh->vertices.assign(tris, tris + 3 * size_t(tri_count));

  std::vector<std::shared_ptr<Material>> materials;
  for(uint32_t i = 0; i < mat_count; ++i) {
    materials.push_back(make_material(mats + 11 * i));
  }
  auto black = std::make_shared<LambertMaterial>(const_texture<Spectrum>(Spectrum(0.f)));

  std::vector<std::unique_ptr<Primitive>> prims;
  std::vector<std::shared_ptr<Light>> lights;
  for(uint32_t i = 0; i < tri_count; ++i) {
    Spectrum le(0.f);
    if(tri_emission) {
      le = Spectrum(tri_emission[3*i], tri_emission[3*i + 1], tri_emission[3*i + 2]);
    }
    if(!le.is_black()) {
      auto shape = std::make_shared<TriangleShape>(mesh.get(), 3 * i);
      auto light = std::make_shared<DiffuseLight>(shape, identity(), le);
      prims.push_back(std::make_unique<ShapePrimitive>(shape, black, light, identity()));
      lights.push_back(light);
    } else {
      uint32_t m = tri_mat ? tri_mat[i] : 0;
      prims.push_back(std::make_unique<TriangleShapePrimitive>(mesh.get(), 3 * i,
            materials.at(m)));
    }
  }

  BvhOpts opts;
  opts.split_method = split_method == 1 ? BvhSplitMethod::Sah : BvhSplitMethod::Middle;
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
  if(bg_const && (bg_const[0] > 0.f || bg_const[1] > 0.f || bg_const[2] > 0.f)) {
    lights.push_back(std::make_shared<InfiniteLight>(
          Spectrum(bg_const[0], bg_const[1], bg_const[2])));
  }
  if(env_rgb && env_w > 0 && env_h > 0) {
    auto img = std::make_shared<Image<PixelRgbFloat>>(env_w, env_h);
    for(uint32_t y = 0; y < env_h; ++y) {
      for(uint32_t x = 0; x < env_w; ++x) {
        const float* p = env_rgb + 3 * (size_t(y) * env_w + x);
        img->set_rgb(x, y, Spectrum(p[0], p[1], p[2]));
      }
    }
    lights.push_back(std::make_shared<EnvironmentLight>(img,
          Spectrum(env_frame[0], env_frame[1], env_frame[2]),
          Vector(env_frame[3], env_frame[4], env_frame[5]),
          Vector(env_frame[6], env_frame[7], env_frame[8])));
  }
  scene->lights = lights;
  for(const auto& light: scene->lights) {
    if(light->flags & LIGHT_BACKGROUND) { scene->background_lights.push_back(light); }
  }
  scene->meshes.push_back(mesh);
  auto t1 = std::chrono::steady_clock::now();
  if(out_build_s) { *out_build_s = std::chrono::duration<double>(t1 - t0).count(); }
  auto* h = new RefPtScene();
  h->scene = scene;
  h->mesh = mesh;
  return h;
}

extern "C" void dref_pt_scene_destroy(void* handle) {
  delete static_cast<RefPtScene*>(handle);
}

extern "C" int dref_pt_scene_render(void* handle,
    const float* cam /* origin, right, up, forward (12 floats) */, float fov,
    uint32_t width, uint32_t height, uint32_t iterations,
    uint32_t min_depth, uint32_t max_depth, int only_direct, int sample_all_lights,
    int strategy /* 0 mis, 1 bsdf, 2 light */, uint32_t seed,
    uint32_t threads, float* out_rgb, double* out_seconds)
{
  auto* h = static_cast<RefPtScene*>(handle);
  auto pool = pool_for(threads);
  CtxG ctx;
  ctx.pool = pool;
  Mat4x4 m(1.f);
  for(int r = 0; r < 3; ++r) {
    m.cols[0][r] = cam[3 + r];
    m.cols[1][r] = cam[6 + r];
    m.cols[2][r] = cam[9 + r];
    m.cols[3][r] = cam[r];
  }
  auto camera = std::make_shared<PinholeCamera>(Transform(m, Mat4x4(1.f)), fov);
  auto film = std::make_shared<Film>(width, height,
      std::make_shared<BoxFilter>(Vec2(0.5f, 0.5f)));
  std::shared_ptr<Sampler> sampler =
    std::make_shared<RandomSampler>(1, Rng(seed))->split(seed);
  PathRenderer::DirectStrategy ds = strategy == 1 ? PathRenderer::DirectStrategy::SAMPLE_BSDF
    : strategy == 2 ? PathRenderer::DirectStrategy::SAMPLE_LIGHT
    : PathRenderer::DirectStrategy::MIS;
  PathRenderer renderer(h->scene, film, sampler, camera, iterations, min_depth, max_depth,
      only_direct != 0, sample_all_lights != 0, ds);
  NoProgress progress;
  auto t0 = std::chrono::steady_clock::now();
  renderer.render(ctx, progress);
  auto t1 = std::chrono::steady_clock::now();
  if(out_seconds) { *out_seconds = std::chrono::duration<double>(t1 - t0).count(); }
  Image<PixelRgbFloat> img = film->to_image<PixelRgbFloat>();
  for(uint32_t y = 0; y < height; ++y) {
    for(uint32_t x = 0; x < width; ++x) {
      PixelRgbFloat p = img.get_pixel(x, y);
      float* o = out_rgb + 3 * (size_t(y) * width + x);
      o[0] = p.r; o[1] = p.g; o[2] = p.b;
    }
  }
  return 0;
}

extern "C" int dref_pt_render(
    const float* verts, uint32_t vert_count, const uint32_t* tris, uint32_t tri_count,
    const uint32_t* tri_mat, const float* mats, uint32_t mat_count,
    const float* tri_emission,
    const float* bg_const, const float* env_rgb, uint32_t env_w, uint32_t env_h,
    const float* env_frame,
    const float* cam, float fov,
    uint32_t width, uint32_t height, uint32_t iterations,
    uint32_t min_depth, uint32_t max_depth, int only_direct, int sample_all_lights,
    int strategy, uint32_t seed, int split_method,
    uint32_t threads, float* out_rgb, double* out_seconds)
{
  void* h = dref_pt_scene_create(verts, vert_count, tris, tri_count, tri_mat, mats, mat_count,
      tri_emission, bg_const, env_rgb, env_w, env_h, env_frame, split_method, threads, nullptr);
  int rc = dref_pt_scene_render(h, cam, fov, width, height, iterations, min_depth, max_depth,
      only_direct, sample_all_lights, strategy, seed, threads, out_rgb, out_seconds);
  dref_pt_scene_destroy(h);
  return rc;
}
