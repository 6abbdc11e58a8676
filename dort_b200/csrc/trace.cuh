// Device ray queries over the wide BVH (bvh_build.h): closest hit and any
// hit.  Shared by the ray-cast kernels and the path tracers.
//
// Replaces Bvh::traverse_elems (src/dort/bvh.cpp:418-469) with the callbacks
// of MeshBvhPrimitive::intersect / intersect_p (mesh_bvh_primitive.cpp:13-45)
// and the triangle tests TriangleUv::hit / Triangle::hit_p
// (triangle.cpp:14-46, 102-134).
//
// Traversal: node groups (base index, 8 child-hit bits << 24 | internal-slot
// mask) on a per-thread stack; child slots are visited in an order fixed by
// the ray octant (slot bit index XOR octant), so no per-node sort is needed.
// Child boxes are tested with fused multiply-adds on the planes (rounded
// outward) and a relative widening that covers the rounding of that
// arithmetic (DG_BOX_HIT); together with the one-step quantization margin the
// test never culls a box containing a hit.
//
// Triangle test: the reference's Moller-Trumbore operations in the
// reference's order with explicit round-to-nearest intrinsics (no fused
// multiply-add, IEEE reciprocal), so (t, b1, b2) are bit-identical to the
// reference computed on the same triangle.
#pragma once
#include <cstdint>
#include <cstring>

#include "common.h"

// The traversal is compiled for the device and, with plain IEEE float
// arithmetic (no contraction), for the host, so that the host can check the
// tree and the traversal without a GPU.
#ifdef __CUDA_ARCH__
#define DG_MUL(a, b) __fmul_rn(a, b)
#define DG_ADD(a, b) __fadd_rn(a, b)
#define DG_SUB(a, b) __fsub_rn(a, b)
#define DG_RCP(a) __frcp_rn(a)
#define DG_U2F(u) __uint2float_rn(u)
#define DG_CLZ(x) __clz(x)
#define DG_POPC(x) __popc(x)
#define DG_FFS(x) __ffs(x)
#define DG_LDG(p) __ldg(p)
#define DG_AS_FLOAT(u) __uint_as_float(u)
#define DG_AS_UINT(f) __float_as_uint(f)
#define DG_BYTE_F(w, j) __uint2float_rn(((w) >> (8 * (j))) & 0xffu)
#define DG_FMA(a, b, c) fmaf(a, b, c)
#define DG_RCP_FAST(a) __frcp_rn(a)
// three-input float max / min (one instruction on sm_100a; exact, like two
// fmaxf / fminf)
__device__ __forceinline__ float dg_max3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float dg_min3(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
#define DG_MAX3(a, b, c) dg_max3(a, b, c)
#define DG_MIN3(a, b, c) dg_min3(a, b, c)
#else
namespace dort_gpu {
inline float host_as_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t host_as_uint(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
}
#define DG_MUL(a, b) ((a) * (b))
#define DG_ADD(a, b) ((a) + (b))
#define DG_SUB(a, b) ((a) - (b))
#define DG_RCP(a) (1.f / (a))
#define DG_U2F(u) (float(u))
#define DG_CLZ(x) __builtin_clz(x)
#define DG_POPC(x) __builtin_popcount(x)
#define DG_FFS(x) __builtin_ffs(int(x))
#define DG_LDG(p) (*(p))
#define DG_AS_FLOAT(u) ::dort_gpu::host_as_float(u)
#define DG_AS_UINT(f) ::dort_gpu::host_as_uint(f)
#define DG_BYTE_F(w, j) (float(((w) >> (8 * (j))) & 0xffu))
#define DG_FMA(a, b, c) std::fma(a, b, c)
#define DG_RCP_FAST(a) (1.f / (a))
#define DG_MAX3(a, b, c) fmaxf(fmaxf(a, b), c)
#define DG_MIN3(a, b, c) fminf(fminf(a, b), c)
#endif
#define DG_HD __host__ __device__ __forceinline__

namespace dort_gpu {

constexpr uint32_t kMiss = 0xffffffffu;
constexpr int kTraceStack = 64;   // == kMaxWideDepth (bvh_build.h)

struct Hit {
  float t, b1, b2;
  uint32_t prim;   // original triangle index, kMiss if none
};

DG_HD float dot_rn(float ax, float ay, float az,
                                        float bx, float by, float bz) {
  // (a.x*b.x + a.y*b.y) + a.z*b.z, each product and sum rounded separately
  return DG_ADD(DG_ADD(DG_MUL(ax, bx), DG_MUL(ay, by)), DG_MUL(az, bz));
}

// Moller-Trumbore as triangle.cpp:109-134 (also 18-42).
DG_HD bool mt_exact(float4 a, float4 e1, float4 e2,
                                         float ox, float oy, float oz,
                                         float dx, float dy, float dz,
                                         float t_min, float t_max,
                                         float& out_t, float& out_b1, float& out_b2) {
  // s1 = cross(dir, e2)
  float s1x = DG_SUB(DG_MUL(dy, e2.z), DG_MUL(dz, e2.y));
  float s1y = DG_SUB(DG_MUL(dz, e2.x), DG_MUL(dx, e2.z));
  float s1z = DG_SUB(DG_MUL(dx, e2.y), DG_MUL(dy, e2.x));
  float det = dot_rn(s1x, s1y, s1z, e1.x, e1.y, e1.z);
  if(det == 0.f) { return false; }
  float inv_det = DG_RCP(det);
  // s = orig - p0
  float sx = DG_SUB(ox, a.x), sy = DG_SUB(oy, a.y), sz = DG_SUB(oz, a.z);
  float b1 = DG_MUL(inv_det, dot_rn(s1x, s1y, s1z, sx, sy, sz));
  if(b1 < 0.f || b1 > 1.f) { return false; }
  // s2 = cross(s, e1)
  float s2x = DG_SUB(DG_MUL(sy, e1.z), DG_MUL(sz, e1.y));
  float s2y = DG_SUB(DG_MUL(sz, e1.x), DG_MUL(sx, e1.z));
  float s2z = DG_SUB(DG_MUL(sx, e1.y), DG_MUL(sy, e1.x));
  float b2 = DG_MUL(inv_det, dot_rn(s2x, s2y, s2z, dx, dy, dz));
  if(b2 < 0.f || DG_ADD(b1, b2) > 1.f) { return false; }
  float t = DG_MUL(inv_det, dot_rn(s2x, s2y, s2z, e2.x, e2.y, e2.z));
  if(t < t_min || t > t_max) { return false; }
  out_t = t;
  out_b1 = b1;
  out_b2 = b2;
  return true;
}

// Moller-Trumbore with fused multiply-adds, for the path tracers (which need
// the reference's estimator, not its rounding).
DG_HD bool mt_fast(float4 a, float4 e1, float4 e2, float ox, float oy, float oz,
                   float dx, float dy, float dz, float t_min, float t_max,
                   float& out_t, float& out_b1, float& out_b2) {
  float s1x = DG_FMA(dy, e2.z, -dz * e2.y);
  float s1y = DG_FMA(dz, e2.x, -dx * e2.z);
  float s1z = DG_FMA(dx, e2.y, -dy * e2.x);
  float det = DG_FMA(s1x, e1.x, DG_FMA(s1y, e1.y, s1z * e1.z));
  if(det == 0.f) { return false; }
  float inv_det = DG_RCP_FAST(det);
  float sx = ox - a.x, sy = oy - a.y, sz = oz - a.z;
  float b1 = inv_det * DG_FMA(s1x, sx, DG_FMA(s1y, sy, s1z * sz));
  if(b1 < 0.f || b1 > 1.f) { return false; }
  float s2x = DG_FMA(sy, e1.z, -sz * e1.y);
  float s2y = DG_FMA(sz, e1.x, -sx * e1.z);
  float s2z = DG_FMA(sx, e1.y, -sy * e1.x);
  float b2 = inv_det * DG_FMA(s2x, dx, DG_FMA(s2y, dy, s2z * dz));
  if(b2 < 0.f || b1 + b2 > 1.f) { return false; }
  float t = inv_det * DG_FMA(s2x, e2.x, DG_FMA(s2y, e2.y, s2z * e2.z));
  if(t < t_min || t > t_max) { return false; }
  out_t = t;
  out_b1 = b1;
  out_b2 = b2;
  return true;
}

// Watertight ray/triangle test: Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013.  The ray's dominant axis
// becomes z and a shear maps the ray onto the z axis; the triangle's edge
// functions U, V, W are then 2-D cross products of the sheared vertices.  An
// edge shared by two triangles gets the same operands in both, so its
// function is computed identically (exactly negated) in both and a ray can
// pass through neither: no leak at edges or vertices.  Products and
// differences are rounded separately (no contraction) so that the negation
// is exact; an edge function that comes out exactly zero is recomputed in
// double.  Barycentrics: b1 = V / det (weight of p1), b2 = W / det (p2).
struct WtRay {
  uint32_t kx, ky, kz;   // dominant axis kz; kx, ky keep the winding
  float sx, sy, sz;      // shear: d[kx] / d[kz], d[ky] / d[kz], 1 / d[kz]
};

DG_HD float wt_sel(float x, float y, float z, uint32_t k) {
  return k == 0 ? x : (k == 1 ? y : z);
}

DG_HD WtRay wt_setup(float dx, float dy, float dz) {
  WtRay r;
  float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
  r.kz = ax > ay ? (ax > az ? 0u : 2u) : (ay > az ? 1u : 2u);
  r.kx = r.kz == 2u ? 0u : r.kz + 1u;
  r.ky = r.kx == 2u ? 0u : r.kx + 1u;
  float dk = wt_sel(dx, dy, dz, r.kz);
  if(dk < 0.f) { uint32_t t = r.kx; r.kx = r.ky; r.ky = t; }
  r.sx = wt_sel(dx, dy, dz, r.kx) / dk;
  r.sy = wt_sel(dx, dy, dz, r.ky) / dk;
  r.sz = 1.f / dk;
  return r;
}

DG_HD bool wt_hit(const WtRay& r, float4 p0, float4 p1, float4 p2, float ox, float oy, float oz,
                  float t_min, float t_max, float& out_t, float& out_b1, float& out_b2) {
  // vertices relative to the origin, permuted (kx, ky, kz)
  float ax = DG_SUB(wt_sel(p0.x, p0.y, p0.z, r.kx), wt_sel(ox, oy, oz, r.kx));
  float ay = DG_SUB(wt_sel(p0.x, p0.y, p0.z, r.ky), wt_sel(ox, oy, oz, r.ky));
  float az = DG_SUB(wt_sel(p0.x, p0.y, p0.z, r.kz), wt_sel(ox, oy, oz, r.kz));
  float bx = DG_SUB(wt_sel(p1.x, p1.y, p1.z, r.kx), wt_sel(ox, oy, oz, r.kx));
  float by = DG_SUB(wt_sel(p1.x, p1.y, p1.z, r.ky), wt_sel(ox, oy, oz, r.ky));
  float bz = DG_SUB(wt_sel(p1.x, p1.y, p1.z, r.kz), wt_sel(ox, oy, oz, r.kz));
  float cx = DG_SUB(wt_sel(p2.x, p2.y, p2.z, r.kx), wt_sel(ox, oy, oz, r.kx));
  float cy = DG_SUB(wt_sel(p2.x, p2.y, p2.z, r.ky), wt_sel(ox, oy, oz, r.ky));
  float cz = DG_SUB(wt_sel(p2.x, p2.y, p2.z, r.kz), wt_sel(ox, oy, oz, r.kz));
  // shear into the ray's frame
  float Ax = DG_SUB(ax, DG_MUL(r.sx, az)), Ay = DG_SUB(ay, DG_MUL(r.sy, az));
  float Bx = DG_SUB(bx, DG_MUL(r.sx, bz)), By = DG_SUB(by, DG_MUL(r.sy, bz));
  float Cx = DG_SUB(cx, DG_MUL(r.sx, cz)), Cy = DG_SUB(cy, DG_MUL(r.sy, cz));
  float U = DG_SUB(DG_MUL(Cx, By), DG_MUL(Cy, Bx));
  float V = DG_SUB(DG_MUL(Ax, Cy), DG_MUL(Ay, Cx));
  float W = DG_SUB(DG_MUL(Bx, Ay), DG_MUL(By, Ax));
  if(U == 0.f || V == 0.f || W == 0.f) {
    U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
    V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
    W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
  }
  if((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) { return false; }
  float det = DG_ADD(DG_ADD(U, V), W);
  if(det == 0.f) { return false; }
  float T = DG_ADD(DG_ADD(DG_MUL(U, DG_MUL(r.sz, az)), DG_MUL(V, DG_MUL(r.sz, bz))),
                   DG_MUL(W, DG_MUL(r.sz, cz)));
  float inv = DG_RCP(det);
  float t = DG_MUL(T, inv);
  if(!(t >= t_min && t <= t_max)) { return false; }
  out_t = t;
  out_b1 = DG_MUL(V, inv);
  out_b2 = DG_MUL(W, inv);
  return true;
}

DG_HD float byte_to_float(uint32_t w, int j) {
  return DG_BYTE_F(w, j);
}

// Widening of the slab test.  The plane distances t carry a relative
// rounding error below 2^-20 of |t| (> 8 ulp).  Widening both ends by that,
// tnear - |tnear| 2^-20 <= tfar + |tfar| 2^-20, takes two fused multiply-adds
// per child; the test used, tnear <= tfar + |tfar| 2^-18, takes one and
// accepts every box the two-sided form accepts, for every sign of tnear and
// tfar (the widening only decides where tnear > tfar: with both >= 0 the
// two-sided form needs tnear <= tfar (1 + 2^-20) / (1 - 2^-20) < tfar (1 +
// 2^-18); with both < 0, |tfar| > |tnear| and 2^-18 |tfar| exceeds the two
// margins together; with tnear >= 0 > tfar both forms reject).
#define DORT_SLAB_FAR_WIDEN 3.814697265625e-6f
#define DG_BOX_HIT(tn, tf) ((tn) <= DG_FMA(fabsf(tf), DORT_SLAB_FAR_WIDEN, (tf)))

// Tests the 8 child boxes of one node; returns the hit mask: bits 24..31 =
// internal children (bit 24 + (slot ^ oct_inv)), bits 0..23 = triangles
// relative to the node's tri_base.
DG_HD uint32_t node_hitmask(
    const uint4& n0, const uint4& n1, const uint4& n2, const uint4& n3, const uint4& n4,
    float ox, float oy, float oz, float ix, float iy, float iz,
    float t_min, float t_max, uint32_t oct_inv4) {
  float px = DG_AS_FLOAT(n0.x), py = DG_AS_FLOAT(n0.y), pz = DG_AS_FLOAT(n0.z);
  float sx = DG_AS_FLOAT((n0.w & 0xffu) << 23);
  float sy = DG_AS_FLOAT(((n0.w >> 8) & 0xffu) << 23);
  float sz = DG_AS_FLOAT(((n0.w >> 16) & 0xffu) << 23);
  float adj_ix = sx * ix, adj_iy = sy * iy, adj_iz = sz * iz;
  float adj_ox = (px - ox) * ix, adj_oy = (py - oy) * iy, adj_oz = (pz - oz) * iz;

  // near / far plane bytes per axis, by direction sign
  const bool nx = ix < 0.f, ny = iy < 0.f, nz = iz < 0.f;
  uint32_t near_x[2] = { nx ? n3.z : n2.x, nx ? n3.w : n2.y };
  uint32_t far_x[2]  = { nx ? n2.x : n3.z, nx ? n2.y : n3.w };
  uint32_t near_y[2] = { ny ? n4.x : n2.z, ny ? n4.y : n2.w };
  uint32_t far_y[2]  = { ny ? n2.z : n4.x, ny ? n2.w : n4.y };
  uint32_t near_z[2] = { nz ? n4.z : n3.x, nz ? n4.w : n3.y };
  uint32_t far_z[2]  = { nz ? n3.x : n4.z, nz ? n3.y : n4.w };

  uint32_t hitmask = 0;
#pragma unroll
  for(int h = 0; h < 2; ++h) {
    uint32_t meta4 = h ? n1.w : n1.z;
    uint32_t is_inner4 = (meta4 & (meta4 << 1)) & 0x10101010u;
    uint32_t inner_mask4 = (is_inner4 >> 4) * 0xffu;
    uint32_t bit_index4 = (meta4 ^ (oct_inv4 & inner_mask4)) & 0x1f1f1f1fu;
    uint32_t child_bits4 = (meta4 >> 5) & 0x07070707u;
#pragma unroll
    for(int j = 0; j < 4; ++j) {
      float tnx = fmaf(byte_to_float(near_x[h], j), adj_ix, adj_ox);
      float tny = fmaf(byte_to_float(near_y[h], j), adj_iy, adj_oy);
      float tnz = fmaf(byte_to_float(near_z[h], j), adj_iz, adj_oz);
      float tfx = fmaf(byte_to_float(far_x[h], j), adj_ix, adj_ox);
      float tfy = fmaf(byte_to_float(far_y[h], j), adj_iy, adj_oy);
      float tfz = fmaf(byte_to_float(far_z[h], j), adj_iz, adj_oz);
      float tnear = DG_MAX3(tnx, tny, fmaxf(tnz, t_min));
      float tfar = DG_MIN3(tfx, tfy, fminf(tfz, t_max));
      bool hit = DG_BOX_HIT(tnear, tfar);
      if(hit) {
        uint32_t bits = (child_bits4 >> (8 * j)) & 0xffu;
        uint32_t bidx = (bit_index4 >> (8 * j)) & 0xffu;
        hitmask |= bits << bidx;
      }
    }
  }
  return hitmask;
}

// Node words per node in device memory: the 224-byte node with float planes
// (bvh_build.h WideNodeF), or in builds with DORT_NODE_QUANTIZED the 80-byte
// quantized node.  The float planes cost 2.8x the node bytes but no
// byte-to-float conversions (48 per node) in the box test, which is issue
// bound: +7 % rays/s on the ray-cast and wavefront workloads.
#ifndef DORT_NODE_QUANTIZED
constexpr uint32_t kNodeWords = 14;
#else
constexpr uint32_t kNodeWords = 5;
#endif

// Child test of a float-plane node (WideNodeF): the same hit mask as
// node_hitmask.  nox = -ox * ix (per ray), so each plane costs one FMA.
DG_HD uint32_t node_hitmask_f(const uint4* np, uint4 h0, float ix, float iy, float iz,
                              float nox, float noy, float noz, float t_min, float t_max,
                              uint32_t oct_inv4) {
  const float4* pl = reinterpret_cast<const float4*>(np + 2);   // [axis][lo, hi][8]
  const int sx = ix < 0.f ? 2 : 0, sy = iy < 0.f ? 2 : 0, sz = iz < 0.f ? 2 : 0;
  uint32_t hitmask = 0;
#pragma unroll
  for(int h = 0; h < 2; ++h) {
    float4 nx = DG_LDG(pl + sx + h), fx = DG_LDG(pl + (2 - sx) + h);
    float4 ny = DG_LDG(pl + 4 + sy + h), fy = DG_LDG(pl + 4 + (2 - sy) + h);
    float4 nz = DG_LDG(pl + 8 + sz + h), fz = DG_LDG(pl + 8 + (2 - sz) + h);
    uint32_t meta4 = h ? h0.w : h0.z;
    uint32_t is_inner4 = (meta4 & (meta4 << 1)) & 0x10101010u;
    uint32_t inner_mask4 = (is_inner4 >> 4) * 0xffu;
    uint32_t bit_index4 = (meta4 ^ (oct_inv4 & inner_mask4)) & 0x1f1f1f1fu;
    uint32_t child_bits4 = (meta4 >> 5) & 0x07070707u;
    const float nxa[4] = {nx.x, nx.y, nx.z, nx.w}, fxa[4] = {fx.x, fx.y, fx.z, fx.w};
    const float nya[4] = {ny.x, ny.y, ny.z, ny.w}, fya[4] = {fy.x, fy.y, fy.z, fy.w};
    const float nza[4] = {nz.x, nz.y, nz.z, nz.w}, fza[4] = {fz.x, fz.y, fz.z, fz.w};
#pragma unroll
    for(int j = 0; j < 4; ++j) {
      float tnear = DG_MAX3(fmaf(nxa[j], ix, nox), fmaf(nya[j], iy, noy),
                            fmaxf(fmaf(nza[j], iz, noz), t_min));
      float tfar = DG_MIN3(fmaf(fxa[j], ix, nox), fmaf(fya[j], iy, noy),
                           fminf(fmaf(fza[j], iz, noz), t_max));
      bool hit = DG_BOX_HIT(tnear, tfar);
      if(hit) {
        uint32_t bits = (child_bits4 >> (8 * j)) & 0xffu;
        uint32_t bidx = (bit_index4 >> (8 * j)) & 0xffu;
        hitmask |= bits << bidx;
      }
    }
  }
  return hitmask;
}

// Traversal state of one ray.  trav_step advances it by one node (the
// node's child boxes, then the triangles of its leaf children); trace_ray
// runs the steps of one ray to the end.  (Handing a finished lane a new ray
// between steps, with a warp vote per step, measured slower than running
// each warp's 32 rays to the end: 1,882 against 2,460 Mrays/s on the ray
// cast at the best threshold, and a slower extension stage at every one.)
struct TravState {
  float ox, oy, oz, dx, dy, dz, t_min;
  float ix, iy, iz;
#ifndef DORT_NODE_QUANTIZED
  float nox, noy, noz;   // -o * inv: one FMA per plane
#endif
  uint32_t oct_inv, oct_inv4;
  WtRay wt;              // the watertight test's ray frame (WT traversals)
  uint2 group;           // current node group: (base, child-hit bits << 24 | internal mask)
  int sp;                // entries on the caller's stack
  Hit best;              // closest hit so far (best.t = t_max while none)
};

DG_HD void trav_init(TravState& s, const TraceScene& sc, float ox, float oy, float oz,
                     float t_min, float dx, float dy, float dz, float t_max) {
  s.ox = ox; s.oy = oy; s.oz = oz; s.dx = dx; s.dy = dy; s.dz = dz; s.t_min = t_min;
  s.best.t = t_max;
  s.best.b1 = 0.f;
  s.best.b2 = 0.f;
  s.best.prim = kMiss;
  // Box-test reciprocals; zero components become tiny so no NaN appears.
  const float tiny = 1e-20f;
  s.ix = 1.f / (fabsf(dx) < tiny ? copysignf(tiny, dx) : dx);
  s.iy = 1.f / (fabsf(dy) < tiny ? copysignf(tiny, dy) : dy);
  s.iz = 1.f / (fabsf(dz) < tiny ? copysignf(tiny, dz) : dz);
  s.oct_inv = (s.ix < 0.f ? 0u : 1u) | (s.iy < 0.f ? 0u : 2u) | (s.iz < 0.f ? 0u : 4u);
  s.oct_inv4 = s.oct_inv * 0x01010101u;
#ifndef DORT_NODE_QUANTIZED
  s.nox = -ox * s.ix;
  s.noy = -oy * s.iy;
  s.noz = -oz * s.iz;
#endif
  s.wt = wt_setup(dx, dy, dz);
  s.sp = 0;
  // root group: internal bit 31 with an empty internal-slot mask -> node 0;
  // an empty tree starts finished
  s.group = make_uint2(0u, sc.node_count ? 0x80000000u : 0u);
}

// Traversal stacks.  A node group is pushed per level descended, so a ray's
// stack holds at most the tree's depth (<= kTraceStack) entries; the trees
// of the benchmark scenes are 8 levels deep.
//
// LocalStack (the default): the stack in per-thread local memory.  Only the
// first few entries are ever touched, and local memory is interleaved so a
// warp's accesses to one depth are coalesced; they stay in the L1 cache.
//
// ShortStack (built with DORT_SHORT_STACK): the first kShortStack entries of
// every thread in shared memory, one column per thread (entry k of thread t
// at k * kShortStackThreads + t: a warp's 8-byte accesses fall in distinct
// banks whatever depth each lane is at), deeper entries in local memory.  It
// measured slower on B200: 598 against 618 M samples/s on the 1080p frame,
// 2,315 against 2,457 Mrays/s on the ray cast, as the shared array takes
// its share of the SM's L1 from the node and triangle fetches.  Blocks wider
// than kShortStackThreads keep the whole stack in local memory.
struct LocalStack {
  uint2 e[kTraceStack];
  DG_HD void init() {}
  DG_HD void push(int sp, uint2 v) { e[sp] = v; }
  DG_HD uint2 pop(int sp) { return e[sp]; }
};

#if defined(__CUDA_ARCH__) && defined(DORT_SHORT_STACK)
constexpr int kShortStack = 8;
constexpr int kShortStackThreads = 128;

// One array per block for every traversal of the kernel (a thread runs one
// traversal at a time).
__device__ __forceinline__ uint2* short_stack_block() {
  __shared__ uint2 s[kShortStack * kShortStackThreads];
  return s;
}

struct ShortStack {
  uint32_t col;        // this thread's column in the block's array
  int lim;             // entries below lim live in shared memory (0: none)
  uint2 deep[kTraceStack];
  __device__ __forceinline__ void init() {
    const uint32_t nt = blockDim.x * blockDim.y * blockDim.z;
    col = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    lim = nt <= kShortStackThreads ? kShortStack : 0;
  }
  __device__ __forceinline__ void push(int sp, uint2 v) {
    if(sp < lim) { short_stack_block()[sp * kShortStackThreads + col] = v; } else { deep[sp] = v; }
  }
  __device__ __forceinline__ uint2 pop(int sp) {
    return sp < lim ? short_stack_block()[sp * kShortStackThreads + col] : deep[sp];
  }
};
using TraceStack = ShortStack;
#else
using TraceStack = LocalStack;
#endif

// Triangle tests of a traversal (WT): kTriMt = Moller-Trumbore on the leaf
// layout (p0, e1, e2), kTriWatertight = wt_hit on the layout (p0, p1, p2) of
// scenes built watertight, kTriByScene = whichever the scene was built for
// (TraceScene::watertight).
enum : int { kTriMt = 0, kTriWatertight = 1, kTriByScene = 2 };

// One traversal step; returns true when the ray is finished (s.best holds
// the closest hit, or for ANY_HIT the first hit found, or prim = kMiss).
template<bool ANY_HIT, bool EXACT_MT, class Stack, int WT = kTriMt>
DG_HD bool trav_step(TravState& s, const TraceScene& sc, Stack& stack) {
  if((s.group.y & 0xff000000u) == 0u) {
    if(s.sp == 0) { return true; }
    s.group = stack.pop(--s.sp);
  }
  uint32_t bit = 31u - DG_CLZ(s.group.y & 0xff000000u);
  s.group.y &= ~(1u << bit);
  uint32_t slot = (bit - 24u) ^ s.oct_inv;
  uint32_t node_idx = s.group.x + DG_POPC(s.group.y & 0xffu & ((1u << slot) - 1u));

  const uint4* np = sc.nodes + kNodeWords * size_t(node_idx);
#ifndef DORT_NODE_QUANTIZED
  uint4 h0 = DG_LDG(np);
  uint32_t imask = DG_LDG(&np[1].x);
  uint32_t hitmask = node_hitmask_f(np, h0, s.ix, s.iy, s.iz, s.nox, s.noy, s.noz, s.t_min,
                                    s.best.t, s.oct_inv4);
  const uint32_t child_base = h0.x, tri_base = h0.y;
#else
  uint4 n0 = DG_LDG(np), n1 = DG_LDG(np + 1), n2 = DG_LDG(np + 2);
  uint4 n3 = DG_LDG(np + 3), n4 = DG_LDG(np + 4);
  uint32_t hitmask = node_hitmask(n0, n1, n2, n3, n4, s.ox, s.oy, s.oz, s.ix, s.iy, s.iz,
                                  s.t_min, s.best.t, s.oct_inv4);
  const uint32_t child_base = n1.x, tri_base = n1.y, imask = n0.w >> 24;
#endif

  uint32_t child_hits = hitmask & 0xff000000u;
  if(child_hits) {
    if(s.group.y & 0xff000000u) {
      // sp < kTraceStack: each push descends one level and the builder
      // bounds the depth by kMaxWideDepth.
      stack.push(s.sp++, s.group);
    }
    s.group = make_uint2(child_base, child_hits | imask);
  }

  uint32_t tri_hits = hitmask & 0x00ffffffu;
  while(tri_hits) {
    uint32_t b = DG_FFS(tri_hits) - 1u;
    tri_hits &= tri_hits - 1u;
    const float4* tp = sc.tris + 3 * size_t(tri_base + b);
    float4 a = DG_LDG(tp), e1 = DG_LDG(tp + 1), e2 = DG_LDG(tp + 2);
    float t, b1, b2;
    bool h;
    if(WT == kTriWatertight || (WT == kTriByScene && sc.watertight)) {
      h = wt_hit(s.wt, a, e1, e2, s.ox, s.oy, s.oz, s.t_min, s.best.t, t, b1, b2);
    } else {
      h = EXACT_MT
          ? mt_exact(a, e1, e2, s.ox, s.oy, s.oz, s.dx, s.dy, s.dz, s.t_min, s.best.t, t, b1, b2)
          : mt_fast(a, e1, e2, s.ox, s.oy, s.oz, s.dx, s.dy, s.dz, s.t_min, s.best.t, t, b1, b2);
    }
    if(h) {
      uint32_t id = DG_AS_UINT(a.w);
      if(ANY_HIT) {
        s.best.t = t; s.best.b1 = b1; s.best.b2 = b2; s.best.prim = id;
        return true;
      }
      if(s.best.prim == kMiss || t < s.best.t || id > s.best.prim) {
        s.best.t = t; s.best.b1 = b1; s.best.b2 = b2; s.best.prim = id;
      }
    }
  }
  return (s.group.y & 0xff000000u) == 0u && s.sp == 0;
}

// Closest hit (ANY_HIT = false) or any hit (ANY_HIT = true) of one ray.
// Returns the hit with prim = kMiss on a miss.  For any hit, prim = the first
// triangle found to intersect.
template<bool ANY_HIT, bool EXACT_MT = true, int WT = kTriMt>
DG_HD Hit trace_ray(const TraceScene& sc, float ox, float oy, float oz, float t_min,
                    float dx, float dy, float dz, float t_max) {
  TravState s;
  trav_init(s, sc, ox, oy, oz, t_min, dx, dy, dz, t_max);
  TraceStack stack;
  stack.init();
  while(!trav_step<ANY_HIT, EXACT_MT, TraceStack, WT>(s, sc, stack)) {}
  return s.best;
}

}  // namespace dort_gpu
