// Device construction of the wide BVH (the format of bvh_build.h).
//
//   1. per-triangle boxes and centroids, centroid bounds (one pass)
//   2. 63-bit Morton codes of the centroids, radix sort (CUB)
//   3. binary tree by Parallel Locally-Ordered Clustering (Meister and
//      Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
//      Hierarchy Construction", IEEE TVCG 2018): each cluster of the
//      Morton-ordered list finds the cluster within 16 positions whose union
//      box has the smallest surface area; mutual nearest neighbours merge;
//      the list is compacted by a prefix sum; repeated until one cluster is
//      left
//   4. top-down collapse into wide nodes, one level per launch pair: a plan
//      pass opens candidates and assigns octant slots (bvh_wide.h, the same
//      functions the host builder uses), a prefix sum of the internal-child
//      and leaf-triangle counts gives every node its child_base / tri_base in
//      breadth-first order, and an emit pass writes the quantized node (or
//      its float-plane form) and the leaf triangles
//
// The result depends only on the input (no atomics decide an order), and
// collapsing the same binary tree on the host gives the same bytes.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "bvh_build.h"

namespace dort_gpu {

enum class DeviceBuilder { kSah, kPloc };

struct DeviceBvh {
  void* nodes = nullptr;          // traversal nodes (WideNodeF, or WideNode when quantized)
  size_t node_bytes = 0;          // allocated bytes of `nodes`
  uint32_t node_count = 0;
  LeafTri* tris = nullptr;        // tri_count leaf triangles
  uint32_t tri_count = 0;
  uint32_t depth = 0;             // levels of wide nodes
  uint32_t iterations = 0;        // SAH levels, or PLOC iterations
  double ms = 0.0;                // wall time of the build (uploads included)
};

// Builds the wide BVH of a host triangle mesh on the current device.  The
// mesh must be valid (indices in range, finite coordinates of magnitude at
// most 1e15: validate_mesh).  On success the caller owns out.nodes and
// out.tris (cudaFree).
bool build_wide_bvh_device(const float* verts, uint32_t vert_count, const uint32_t* tris,
                           uint32_t tri_count, const BuildOptions& opts, DeviceBuilder method,
                           cudaStream_t stream, DeviceBvh& out, std::string& err,
                           BinaryDump* dump = nullptr);

}  // namespace dort_gpu
