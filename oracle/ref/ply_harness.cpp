// PLY ingest harness around the reference renderer's reader.
//
// TEST INFRASTRUCTURE ONLY: compiled with the reference's ply_mesh.cpp and
// the rply library it vendors by oracle/Makefile into oracle/_ref/.  Reads a
// PLY file with read_ply_to_mesh (src/dort/ply_mesh.cpp:80-102, identity
// transform) so that the tests can compare the product's readers (the Lua
// front-end's and dort_b200.builder's) with the reference's points and
// triangle fan.  Nothing in the product links it.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "dort/mesh.hpp"
#include "dort/ply_mesh.hpp"
#include "dort/transform.hpp"

// Returns 0 and fills counts = {points, vertex indices} on success (arrays
// are written only up to their capacities), -1 if the file cannot be opened,
// -2 if the reader fails.
extern "C" int dref_read_ply(const char* path, float* points, uint32_t max_points,
                             uint32_t* vertices, uint32_t max_vertices, uint32_t* counts) {
  FILE* file = std::fopen(path, "rb");
  if(!file) { return -1; }
  dort::Mesh mesh;
  bool ok = dort::read_ply_to_mesh(file, dort::identity(), mesh, [](uint32_t) {});
  std::fclose(file);
  if(!ok) { return -2; }
  counts[0] = uint32_t(mesh.points.size());
  counts[1] = uint32_t(mesh.vertices.size());
  for(uint32_t i = 0; i < counts[0] && i < max_points; ++i) {
    points[3 * i + 0] = mesh.points[i].v.x;
    points[3 * i + 1] = mesh.points[i].v.y;
    points[3 * i + 2] = mesh.points[i].v.z;
  }
  for(uint32_t i = 0; i < counts[1] && i < max_vertices; ++i) {
    vertices[i] = mesh.vertices[i];
  }
  return 0;
}
