// Host emulation of the device ray query: builds the same wide BVH the
// device scene uses and runs the same traversal code (trace.cuh compiled for
// the host) on the CPU.  It lets the builder, the quantization and the
// traversal be checked without a GPU; it is not a fallback for the device
// path (nothing routes device work here).
#include <string>
#include <vector>

#include "bvh_build.h"
#include "common.h"
#include "trace.cuh"

using namespace dort_gpu;

extern "C" int dort_gpu_host_check_raycast(const dort_scene_desc* desc, const float* rays,
                                           size_t ray_count, int any_hit,
                                           uint32_t* out_prim, float* out_tb,
                                           uint32_t* out_depth) try {
  clear_error();
  if(!desc || (ray_count && (!rays || !out_prim || (!any_hit && !out_tb)))) {
    return fail(DORT_ERR_INVALID, "null argument");
  }
  if(desc->struct_size != sizeof(dort_scene_desc)) {
    return fail(DORT_ERR_INVALID, "dort_scene_desc.struct_size mismatch (ABI version)");
  }
  BuildOptions opts;
  opts.width = desc->bvh_width ? desc->bvh_width : 8;
  WideBvh bvh;
  std::string err;
  if(!build_wide_bvh(desc->verts, desc->vert_count, desc->tris, desc->tri_count, opts,
                     bvh, err)) {
    return fail(DORT_ERR_INVALID, err);
  }
  const bool wt = (desc->flags & DORT_SCENE_WATERTIGHT) != 0;
  if(wt) {
    // the leaf layout of watertight scenes: the three input vertices
    for(LeafTri& lt : bvh.tris) {
      for(int k = 0; k < 3; ++k) {
        const float* p = desc->verts + 3 * size_t(desc->tris[3 * size_t(lt.id) + k]);
        float* dst = k == 0 ? lt.p0 : (k == 1 ? lt.e1 : lt.e2);
        dst[0] = p[0]; dst[1] = p[1]; dst[2] = p[2];
      }
    }
  }
  TraceScene sc;
  sc.nodes = reinterpret_cast<const uint4*>(traversal_nodes(bvh));
  sc.tris = reinterpret_cast<const float4*>(bvh.tris.data());
  sc.node_count = uint32_t(bvh.nodes.size());
  sc.tri_count = uint32_t(bvh.tris.size());
  sc.watertight = wt ? 1u : 0u;
  if(out_depth) { *out_depth = bvh.depth; }
  for(size_t i = 0; i < ray_count; ++i) {
    const float* r = rays + 8 * i;
    Hit h = any_hit
        ? (wt ? trace_ray<true, true, kTriWatertight>(sc, r[0], r[1], r[2], r[3], r[4], r[5],
                                                      r[6], r[7])
              : trace_ray<true>(sc, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]))
        : (wt ? trace_ray<false, true, kTriWatertight>(sc, r[0], r[1], r[2], r[3], r[4], r[5],
                                                       r[6], r[7])
              : trace_ray<false>(sc, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]));
    if(any_hit) {
      out_prim[i] = h.prim != kMiss ? 1u : 0u;
    } else {
      out_prim[i] = h.prim;
      if(h.prim != kMiss) {
        out_tb[3 * i] = h.t;
        out_tb[3 * i + 1] = h.b1;
        out_tb[3 * i + 2] = h.b2;
      }
    }
  }
  return DORT_OK;
} DORT_ABI_CATCH
