// The adjoint's term log: what one sample's path contributed, recorded while
// the path is traced and turned into gradients once the sample's value L is
// known (adjoint.cu: one thread per sample with the log in local memory;
// wavefront.cu: the log per path slot in device memory, written by the
// shade, shadow and BSDF-strategy stages and applied by the regeneration
// stage when the sample ends).
//
// Entries are float4 (x, y, z, tag), tag = kind << 30 | primitive:
//   kEvEmission  (thr)      a path hit an emitting triangle: dL/dLe += thr
//   kEvDirect    (c)        a direct-lighting term c from a light triangle:
//                           dL/dLe += c / Le
//   kEvVertex    (A), (a)   two entries: a Lambert vertex, the sum A of the
//                           terms before it and its albedo a; every later
//                           term is linear in a: dL/da += (L - A) / a
// (per colour channel, each weighted by dLoss/dI(pixel) / spp).
#pragma once
#include "pt.cuh"

namespace dort_gpu {

constexpr uint32_t kAdjLog = 32;   // entries per sample
enum : uint32_t { kEvEmission = 0u, kEvDirect = 1u, kEvVertex = 2u };
constexpr uint32_t kEvPrimMask = (1u << 30) - 1u;

DG_HD float4 adj_entry(uint32_t kind, uint32_t prim, V3 v) {
  return make_float4(v.x, v.y, v.z, DG_AS_FLOAT(kind << 30 | prim));
}

// Applies n recorded entries (entry k at ev[k * stride]) of a sample of value
// L with image weight adj.
__device__ __forceinline__ void adj_apply(const float4* ev, size_t stride, uint32_t n, V3 L,
                                          V3 adj, const float* tri_emission, float* d_albedo,
                                          float* d_emission) {
  for(uint32_t i = 0; i < n; ++i) {
    const float4 e = ev[i * stride];
    const uint32_t tag = DG_AS_UINT(e.w), kind = tag >> 30;
    const size_t prim = tag & kEvPrimMask;
    if(kind == kEvEmission) {
      float* g = d_emission + 3 * prim;
      atomicAdd(g, adj.x * e.x);
      atomicAdd(g + 1, adj.y * e.y);
      atomicAdd(g + 2, adj.z * e.z);
    } else if(kind == kEvDirect) {
      const float* le = tri_emission + 3 * prim;
      float* g = d_emission + 3 * prim;
      if(le[0] > 0.f) { atomicAdd(g, adj.x * e.x / le[0]); }
      if(le[1] > 0.f) { atomicAdd(g + 1, adj.y * e.y / le[1]); }
      if(le[2] > 0.f) { atomicAdd(g + 2, adj.z * e.z / le[2]); }
    } else {
      const float4 c = ev[++i * stride];
      const V3 rem = L - v3(e.x, e.y, e.z);
      float* g = d_albedo + 3 * prim;
      if(c.x > 0.f) { atomicAdd(g, adj.x * rem.x / c.x); }
      if(c.y > 0.f) { atomicAdd(g + 1, adj.y * rem.y / c.y); }
      if(c.z > 0.f) { atomicAdd(g + 2, adj.z * rem.z / c.z); }
    }
  }
}

// A sample the film keeps (renderer.cpp:36-41); others have no gradient.
DG_HD bool adj_kept(V3 L) {
  return isfinite(L.x) && isfinite(L.y) && isfinite(L.z) && L.x >= 0.f && L.y >= 0.f &&
         L.z >= 0.f;
}

// Does a vertex with material m and primitive tri record an albedo entry?
DG_HD bool adj_albedo_vertex(const DevMaterial& m, uint32_t tri, uint32_t tri_count) {
  return m.kind == DORT_MAT_LAMBERT && m.bxdf_flags != 0u && tri < tri_count;
}

}  // namespace dort_gpu
