// Host-side BVH construction for the device scene.
//
// The reference builds a binary BVH per mesh with middle or SAH splits
// (src/dort/bvh.cpp:9-416) and traverses it with a 64-entry stack of 32-byte
// nodes (bvh.cpp:418-469).  The device scene instead uses a wide BVH (up to 8
// children per node) with 8-bit quantized child boxes and octant-ordered
// child slots, laid out for 128-bit loads:
//
//   WideNode (80 bytes = 5 x uint4, 16-byte aligned, always 3 x 32-byte
//   sectors):
//     float    p[3]        origin of the quantization grid
//     uint8_t  e[3]        biased power-of-two exponents of the grid step
//     uint8_t  imask       bit s set: slot s is an internal child
//     uint32_t child_base  node index of the first internal child; internal
//                          children are contiguous, ordered by slot
//     uint32_t tri_base    index of the node's first triangle
//     uint8_t  meta[8]     per slot: 0 = empty; internal: 0x20 | (24 + s);
//                          leaf: (unary triangle count << 5) | tri offset
//     uint8_t  qlo[3][8], qhi[3][8]   quantized child boxes
//
// Child boxes are quantized outward with one full grid step of margin on
// every side, so that the device slab test (rounded float arithmetic) never
// culls a child that contains a hit.  The device traverses WideNodeF (below):
// the same nodes with those quantized planes expanded to floats.
//
//   Triangle (48 bytes = 3 x float4, leaf order):
//     (p0.xyz, original triangle index as bits), (e1.xyz, 0), (e2.xyz, 0)
//   with e1 = p1 - p0 and e2 = p2 - p0 rounded exactly as the reference does
//   inside Triangle::hit_p (triangle.cpp:18-19).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dort_gpu {

// Throws std::bad_alloc when a test's injected allocation failure is due
// (dort_gpu_debug_fail_alloc); called before the builders' large allocations.
void alloc_checkpoint();


struct alignas(16) WideNode {
  float p[3];
  uint8_t e[3];
  uint8_t imask;
  uint32_t child_base;
  uint32_t tri_base;
  uint8_t meta[8];
  uint8_t qlo[3][8];
  uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

// The same node with float child planes: the quantized planes p + s q of
// every child (margin included) rounded outward to float, so the device box
// test needs no byte-to-float conversion.  224 bytes = 14 x uint4.
struct alignas(16) WideNodeF {
  uint32_t child_base;
  uint32_t tri_base;
  uint8_t meta[8];
  uint32_t imask;
  uint32_t pad[3];
  float pl[3][2][8];   // [axis][0: lo, 1: hi][slot]
};
static_assert(sizeof(WideNodeF) == 224, "WideNodeF must be 224 bytes");

// Expands quantized nodes into WideNodeF.
void expand_node_planes(const std::vector<WideNode>& in, std::vector<WideNodeF>& out);

struct alignas(16) LeafTri {
  float p0[3];
  uint32_t id;
  float e1[3];
  float pad1;
  float e2[3];
  float pad2;
};
static_assert(sizeof(LeafTri) == 48, "LeafTri must be 48 bytes");

// Cost of a traversal step relative to a triangle test in the binary SAH of
// both builders (host and device build the same tree).
constexpr double kSahTraversal = 0.5;

struct BuildOptions {
  uint32_t width = 8;          // children per node, 2..8
  uint32_t max_leaf_tris = 2;  // triangles per leaf slot, 1..3 (2: +2.7 % on the ray cast)
  uint32_t bins = 32;          // SAH bins per axis
  uint32_t threads = 0;        // 0: hardware concurrency
};

struct WideBvh {
  std::vector<WideNode> nodes;
  std::vector<WideNodeF> nodes_f;   // float-plane nodes (traversed unless DORT_NODE_QUANTIZED)
  std::vector<LeafTri> tris;
  uint32_t depth = 0;          // levels of wide nodes
  double root_lo[3] = {0, 0, 0};
  double root_hi[3] = {0, 0, 0};
};

// The node array the device traversal reads, and its size in bytes.
inline const void* traversal_nodes(const WideBvh& b) {
#ifndef DORT_NODE_QUANTIZED
  return b.nodes_f.data();
#else
  return b.nodes.data();
#endif
}
inline size_t traversal_node_bytes(const WideBvh& b) {
#ifndef DORT_NODE_QUANTIZED
  return b.nodes_f.size() * sizeof(WideNodeF);
#else
  return b.nodes.size() * sizeof(WideNode);
#endif
}

// Maximum stack depth the device traversal supports; the builder guarantees
// that no root-to-leaf path of the wide tree is deeper.
constexpr uint32_t kMaxWideDepth = 64;

// The binary tree the device made, for checks.  A leaf has bit 31 set in
// `left`, the rest of `left` is its first position in leaf_idx and `right`
// its triangle count; an internal node has its children in left / right.
// count = triangles below each node.
struct BinaryDump {
  std::vector<float> lo, hi;      // 3 per node
  std::vector<uint32_t> left, right, count;
  std::vector<uint32_t> leaf_idx;    // triangle indices in leaf order
  uint32_t root = 0;
};

// Collapses a binary tree made elsewhere (the device builder's) with the
// host's collapse, for checking the device collapse byte for byte.
bool collapse_binary_dump(const BinaryDump& tree, const float* verts, const uint32_t* tris,
                          uint32_t tri_count, const BuildOptions& opts, WideBvh& out,
                          std::string& err);

// Surface-area cost of a wide BVH from its float planes, relative to the
// root box: sum over visited child nodes of area, plus sum over leaf slots of
// area x triangle count (traversal and intersection cost 1 each).
double wide_sah_cost(const WideNodeF* nodes, size_t node_count);

// The input checks of build_wide_bvh, with the same messages (indices in
// range, finite coordinates of magnitude at most 1e15).
bool validate_mesh(const float* verts, uint32_t vert_count, const uint32_t* tris,
                   uint32_t tri_count, std::string& err);

// Builds the wide BVH; returns false (with a message) on invalid input.
bool build_wide_bvh(const float* verts, uint32_t vert_count,
                    const uint32_t* tris, uint32_t tri_count,
                    const BuildOptions& opts, WideBvh& out, std::string& err);

}  // namespace dort_gpu
