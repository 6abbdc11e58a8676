// Ray-cast harness around the reference renderer's own BVH and triangle code.
//
// TEST INFRASTRUCTURE ONLY: this file is compiled together with the
// reference's sources (src/dort/bvh.cpp, box.cpp, triangle.cpp,
// thread_pool.cpp, stats.cpp) by oracle/Makefile into oracle/_ref/.  It is
// used to pin the C restatement in oracle/raycast.c and as the CPU baseline
// ("reference" kind) for the ray-cast workload.  Nothing in the product links
// it.
//
// The reference has no API that casts a single ray and reports the hit
// triangle index (MeshBvhPrimitive hides it), so this harness instantiates the
// reference's Bvh template with the same traits MeshBvhPrimitive uses
// (mesh_bvh_primitive.hpp:9-16: Element = vertex-array offset, bounds =
// Triangle(mesh, idx).bounds()) and replays MeshBvhPrimitive::intersect /
// intersect_p (mesh_bvh_primitive.cpp:13-45) while recording the index.
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>
#include "dort/bvh.hpp"
#include "dort/mesh.hpp"
#include "dort/shape.hpp"
#include "dort/thread_pool.hpp"
#include "dort/triangle.hpp"

// The template definitions of Bvh<> live in the reference's .cpp file.
#include "dort/bvh.cpp"  // found through -I<reference>/src

namespace {
  struct HarnessTraits {
    using Element = uint32_t;
    using Arg = const dort::Mesh*;
    static dort::Box get_bounds(const dort::Mesh* mesh, uint32_t idx) {
      return dort::Triangle(*mesh, idx).bounds();
    }
  };
}

template class dort::Bvh<HarnessTraits>;

namespace {
  struct RefScene {
    dort::Mesh mesh;
    std::unique_ptr<dort::Bvh<HarnessTraits>> bvh;
  };

  dort::ThreadPool& pool_with(uint32_t threads) {
    static dort::ThreadPool pool;
    static uint32_t started = 0;
    if(started != threads) {
      if(started != 0) { pool.stop(); }
      pool.start(threads);
      started = threads;
    }
    return pool;
  }

  double now_s() {
    return std::chrono::duration<double>(
        std::chrono::steady_clock::now().time_since_epoch()).count();
  }
}

extern "C" {

// Builds the reference BVH over a triangle mesh.  split_method: 0 = middle
// (reference default), 1 = SAH.  Returns an opaque handle.
void* dref_scene_create(const float* verts, uint32_t vert_count,
    const uint32_t* tri_idx, uint32_t tri_count, int split_method,
    uint32_t leaf_size, uint32_t max_leaf_size, uint32_t threads,
    double* out_build_s)
{
  auto* scene = new RefScene();
  scene->mesh.points.reserve(vert_count);
  for(uint32_t i = 0; i < vert_count; ++i) {
    scene->mesh.points.push_back(dort::Point(
          verts[3*i], verts[3*i + 1], verts[3*i + 2]));
  }
  scene->mesh.vertices.assign(tri_idx, tri_idx + 3*size_t(tri_count));

  std::vector<uint32_t> elems(tri_count);
  for(uint32_t i = 0; i < tri_count; ++i) { elems[i] = 3*i; }

  dort::BvhOpts opts;
  opts.split_method = split_method == 1
    ? dort::BvhSplitMethod::Sah : dort::BvhSplitMethod::Middle;
  opts.leaf_size = leaf_size;
  opts.max_leaf_size = max_leaf_size;

  // The reference's ThreadPool is only safe with one worker: with more, a
  // thread can read a finished loop's flags after its owner returned
  // (thread_pool.cpp:112-148) and crash.  The build runs on one worker.
  (void)threads;
  double t0 = now_s();
  scene->bvh = std::make_unique<dort::Bvh<HarnessTraits>>(
      std::move(elems), &scene->mesh, opts, pool_with(1));
  if(out_build_s) { *out_build_s = now_s() - t0; }
  return scene;
}

void dref_scene_destroy(void* handle) {
  delete static_cast<RefScene*>(handle);
}

// Casts rays (8 floats each: orig.xyz, t_min, dir.xyz, t_max).  Closest hit
// writes out_prim[i] = triangle index or 0xffffffff, out_tb[3i..3i+2] =
// (t, b1, b2); any hit writes out_prim[i] = 1/0 and leaves out_tb untouched.
// out_tests (optional) receives the number of triangle tests per ray.
int dref_raycast(void* handle, const float* rays, uint64_t ray_count,
    int any_hit, uint32_t threads, uint32_t* out_prim, float* out_tb,
    uint32_t* out_tests, double* out_trace_s)
{
  auto* scene = static_cast<RefScene*>(handle);
  const uint64_t chunk = 4096;
  uint32_t jobs = uint32_t((ray_count + chunk - 1) / chunk);

  // Rays are spread over plain threads of this harness (see the note on the
  // reference's ThreadPool in dref_scene_create); each ray runs the
  // reference's own traversal.
  std::atomic<uint32_t> next_job{0};
  auto run_job = [&](uint32_t job) {
    uint64_t begin = uint64_t(job) * chunk;
    uint64_t end = std::min(ray_count, begin + chunk);
    for(uint64_t i = begin; i < end; ++i) {
      const float* r = rays + 8*i;
      dort::Ray ray(dort::Point(r[0], r[1], r[2]),
          dort::Vector(r[4], r[5], r[6]), r[3], r[7]);
      uint32_t tests = 0;
      if(any_hit) {
        bool found = false;
        scene->bvh->traverse_elems(ray, [&](uint32_t index) {
          tests += 1;
          if(dort::Triangle(scene->mesh, index).hit_p(ray)) {
            found = true;
            return false;
          }
          return true;
        });
        out_prim[i] = found ? 1u : 0u;
      } else {
        bool found = false;
        uint32_t hit_index = 0;
        float hit_t = 0.f;
        dort::DiffGeom hit_geom;
        scene->bvh->traverse_elems(ray, [&](uint32_t index) {
          tests += 1;
          float t_hit;
          float ray_epsilon;
          dort::DiffGeom geom;
          if(dort::TriangleUv(scene->mesh, index).hit(ray, t_hit,
                ray_epsilon, geom)) {
            found = true;
            ray.t_max = t_hit;
            hit_index = index;
            hit_t = t_hit;
            hit_geom = geom;
          }
          return true;
        });
        if(found) {
          out_prim[i] = hit_index / 3;
          // With the default uvs (0,0),(1,0),(0,1) (triangle.cpp:89-93) the
          // interpolated uv equals the barycentrics (b1, b2) exactly.
          out_tb[3*i + 0] = hit_t;
          out_tb[3*i + 1] = hit_geom.uv.x;
          out_tb[3*i + 2] = hit_geom.uv.y;
        } else {
          out_prim[i] = 0xffffffffu;
        }
      }
      if(out_tests) { out_tests[i] = tests; }
    }
  };
  double t0 = now_s();
  uint32_t nthreads = threads > 0 ? threads : 1;
  std::vector<std::thread> workers;
  for(uint32_t t = 0; t < nthreads; ++t) {
    workers.emplace_back([&]() {
      for(uint32_t job = next_job.fetch_add(1); job < jobs; job = next_job.fetch_add(1)) {
        run_job(job);
      }
    });
  }
  for(auto& w : workers) { w.join(); }
  if(out_trace_s) { *out_trace_s = now_s() - t0; }
  return 0;
}

}
