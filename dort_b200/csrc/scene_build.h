// Host-side assembly of a renderable scene from a dort_scene_desc: the wide
// BVH plus the shading tables the path tracer reads.  The same host arrays are
// uploaded for the device and used directly by the host checks.
#pragma once
#include <string>
#include <vector>

#include "bvh_build.h"
#include "pt_scene.h"

namespace dort_gpu {

struct HostScene {
  WideBvh bvh;                       // empty when device_bvh (built on the device)
  bool device_bvh = false;
  double bvh_ms = 0.0;               // host BVH build time
  std::vector<float4> shade;         // 3 per triangle
  std::vector<DevMaterial> mats;
  std::vector<DevLight> lights;
  std::vector<float> light_cdf;
  uint32_t bg_count = 0;
  uint32_t bg_light[2] = {0, 0};
  std::vector<float> env_rgb, env_pdfs;
  std::vector<float2> env_row_alias, env_col_alias;
  std::vector<DevShape> shapes;
  std::vector<DevShape> light_shapes;
  uint32_t general = 0;   // needs the general path instantiation (pt.cuh)
  uint32_t shape_base = 0;
  DevEnv env{};
  uint32_t emissive_count = 0;
  float radius = 0.f;
  float centroid[3] = {0.f, 0.f, 0.f};
};

// The device form of one material (validated; false + message on error).
bool material_to_device(const dort_material& in, DevMaterial& m, std::string& err);

// Analytic shapes are intersected as a list after the BVH.
constexpr uint32_t kMaxShapes = 4096;

// Validates the description and builds everything; false + message on error.
// With allow_device_bvh and a description that asks for the device build
// (bvh_build DEFAULT or DEVICE) the mesh is only validated and hs.bvh stays
// empty: the caller builds the BVH on the device.
bool build_host_scene(const dort_scene_desc* desc, HostScene& out, std::string& err,
                      bool allow_device_bvh = false);

// Device-view structures pointing at the host arrays (host checks only).
PtScene host_view(const HostScene& hs);

}  // namespace dort_gpu
