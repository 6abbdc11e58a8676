// Device view of a renderable scene and of the render parameters.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dort_gpu.h"

namespace dort_gpu {

// Device view of the ray-query part of a scene.
struct TraceScene {
  const uint4* nodes;   // 5 x uint4 per WideNode (bvh_build.h)
  const float4* tris;   // 3 x float4 per LeafTri
  uint32_t node_count;
  uint32_t tri_count;
  uint32_t watertight;  // leaf triangles hold (p0, p1, p2) for the watertight test
};

// BxDF flag bits as the reference's BxdfFlags (include/dort/bsdf.hpp:8-28).
enum : uint32_t {
  F_REFL = 1, F_TRANS = 2, F_DIFF = 4, F_GLOSSY = 8, F_DELTA = 16,
  F_MODES = F_REFL | F_TRANS, F_LOBES = F_DIFF | F_GLOSSY | F_DELTA,
  F_ALL = F_MODES | F_LOBES,
};

// Resolved material: which single BxDF the reference's Material::add_bxdfs
// would add (every material in scope adds at most one), with its constants.
struct DevMaterial {
  uint32_t kind;      // DORT_MAT_* ; bxdf_flags == 0: no BxDF (black)
  uint32_t bxdf_flags;
  float c[3];         // lambert/mirror albedo; dielectric reflect tint;
                      // phong diffuse; conductor F0
  float c2[3];        // dielectric transmit tint; phong glossy
  float p0;           // dielectric ior_inside; phong exponent; conductor alpha
  float p1;           // phong: glossy sampling weight
  float p2, p3;
};

enum : uint32_t {
  LIGHT_TRI = 0, LIGHT_INFINITE = 1, LIGHT_ENV = 2,
  LIGHT_SHAPE = 3,    // DiffuseLight on an analytic shape (sphere or disk)
  LIGHT_POINT = 4, LIGHT_DIR = 5,
};

struct DevLight {
  uint32_t kind;
  uint32_t tri;       // LIGHT_TRI: original triangle index; LIGHT_SHAPE: light_shapes index
  float L[3];         // radiance (point: intensity; LIGHT_ENV: unused)
  float area;         // LIGHT_TRI: triangle area; LIGHT_SHAPE: area in shape space
  float p0[3], e1[3], e2[3];   // LIGHT_POINT: p0 = position
  float nn[3];        // LIGHT_TRI: normalize(cross(e2, e1)); LIGHT_DIR: unit direction
};

enum : uint32_t { SHAPE_SPHERE = 1, SHAPE_DISK = 2, SHAPE_CUBE = 3, SHAPE_CYLINDER = 4 };

// Analytic shape primitive: shape parameters, material, optional area light
// and the shape-to-world transform with its inverse (3x4 row-major each).
struct DevShape {
  uint32_t kind;
  uint32_t mat;
  uint32_t light;     // light index + 1, 0 if not emissive
  float r, z0, z1;    // sphere: r; disk: r, z0; cylinder: r, z0 = z_min, z1 = z_max
  float m[12];        // shape to world
  float inv[12];      // world to shape
};

// Latitude-longitude environment map (EnvironmentLight,
// environment_light.cpp:6-158) with its piecewise-constant 2-D distribution
// (piecewise_distrib_2d.cpp).
struct DevEnv {
  const float* rgb;          // w * h * 3
  const float* pdfs;         // w * h
  // the same distribution as alias tables: rows (h entries), then the
  // columns of each row (w * h); (probability, alias index as float bits)
  const float2* row_alias;
  const float2* col_alias;
  uint32_t w, h;
  float scale[3];
  float up[3], s[3], t[3];
};

struct PtScene {
  TraceScene trace;
  const float4* shade;       // 3 per original triangle: (p0, material), (p1, light+1), (p2, 0)
  const DevMaterial* mats;
  uint32_t mat_count;
  const float* tri_albedo;   // optional per-triangle albedo override (tri_count * 3)
  const float* tri_emission; // optional per-triangle emission override (tri_count * 3)
  const DevLight* lights;
  uint32_t light_count;
  const float* light_cdf;    // light_count + 1
  uint32_t bg_count;
  uint32_t bg_light[2];      // indices into lights of the background lights
  DevEnv env;
  const DevShape* shapes;    // analytic shapes; hit prim = shape_base + index
  uint32_t shape_count;
  uint32_t shape_base;       // number of triangles
  const DevShape* light_shapes;  // the shapes of LIGHT_SHAPE lights, under the
                                 // lights' own transforms
  uint32_t general;          // 1 if the scene has analytic shapes, delta lights,
                             // Oren-Nayar or a general dielectric (host use)
  float centroid[3];         // Scene::centroid / radius: the bounds' centre and
  float radius;              // half diagonal (distant lights start on its disk)
};

enum : uint32_t { CAMERA_PINHOLE = 0, CAMERA_ORTHO = 1, CAMERA_THIN_LENS = 2 };

struct PtParams {
  float origin[3], right[3], up[3], forward[3];
  float proj_dim;            // 2 tan(fov / 2) (pinhole, thin lens)
  uint32_t camera;           // CAMERA_*
  float lens_radius, focal_distance;
  float ortho_dim;           // orthographic image plane dimension
  uint32_t width, height;
  uint32_t spp;              // iterations
  uint32_t min_depth, max_depth;
  uint32_t only_direct, sample_all_lights;
  uint32_t strategy;         // 0 mis, 1 bsdf, 2 light
  uint64_t seed;
  uint32_t renderer;         // RENDERER_PT, RENDERER_LT, RENDERER_BDPT
  float cam_inv[9];          // rows of [right up forward]^-1 (world to camera)
  uint32_t use_t1;           // bdpt: connect light subpaths to the camera (t = 1)
  uint32_t roulette;         // pt: Russian roulette after bounce 2 (the reference's rule)
};

enum : uint32_t { RENDERER_PT = 0, RENDERER_LT = 1, RENDERER_BDPT = 2 };

// Whether rendering `sc` with `pp` needs the general instantiation of the
// path code (pt.cuh, template flag G).
inline bool scene_needs_general(const PtScene& sc, const PtParams& pp) {
  return sc.general != 0 || pp.camera != CAMERA_PINHOLE || sc.trace.watertight != 0 ||
         pp.sample_all_lights != 0;
}

}  // namespace dort_gpu
