/* Test oracle for the dort ray-cast and path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement, in plain C, of the
 * reference renderer's algorithms (honzasp/dort).  Only the test suite, the
 * smoke check and the CPU-baseline leg of the benchmark call it, and only as
 * the checker; the product library never links or loads it.
 *
 * Every function cites the reference file:line it restates.  Parity of the
 * restatement itself is pinned against the reference compiled from its own
 * sources (oracle/_ref/libdort_ref.so, built by oracle/Makefile) and against
 * golden vectors committed under tests/golden/.
 */
#ifndef DORT_ORACLE_H
#define DORT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_bvh orc_bvh;

/* Binary BVH over a triangle mesh, built exactly as Bvh<>::Bvh
 * (bvh.cpp:9-55).  split_method: 0 = middle (reference default), 1 = SAH. */
orc_bvh* orc_bvh_build(const float* verts, uint32_t vert_count,
    const uint32_t* tri_idx, uint32_t tri_count, int split_method,
    uint32_t leaf_size, uint32_t max_leaf_size);
void orc_bvh_free(orc_bvh* bvh);
uint32_t orc_bvh_node_count(const orc_bvh* bvh);
/* Depth-first dump: per node (lo.xyz, hi.xyz) and (offset_or_left, count,
 * axis); lets tests compare topologies. */
void orc_bvh_nodes(const orc_bvh* bvh, float* boxes, uint32_t* meta);

/* Ray layout: 8 floats per ray (orig.xyz, t_min, dir.xyz, t_max).
 * Closest hit (any_hit = 0): out_prim = triangle index or 0xffffffff,
 * out_tb = (t, b1, b2).  Any hit: out_prim = 1 (occluded) / 0.
 * out_nodes / out_tests (optional) count visited nodes and triangle tests,
 * the algorithmic work per ray (bvh.cpp:432, triangle.cpp:105). */
void orc_raycast(const orc_bvh* bvh, const float* rays, uint64_t ray_count,
    int any_hit, uint32_t* out_prim, float* out_tb,
    uint32_t* out_nodes, uint32_t* out_tests);

/* Brute-force closest hit over all triangles with the same arithmetic, used
 * to classify disagreements. */
void orc_raycast_brute(const float* verts, const uint32_t* tri_idx,
    uint32_t tri_count, const float* rays, uint64_t ray_count,
    uint32_t* out_prim, float* out_tb);

/* The reference's Moller-Trumbore test (triangle.cpp:102-134) on one
 * triangle; returns 1 on hit and writes (t, b1, b2). */
int orc_triangle_hit(const float* p0, const float* p1, const float* p2,
    const float* ray, float* out_tb);

/* Float64 "pt" estimator and its gradient (pt64.c) on Lambert triangle
 * scenes with triangle emitters and a pinhole camera, using the device's
 * random-number streams.  albedo / emission: tri_count * 3 (the values in
 * effect); light_power_emission: the emission the scene was created with
 * (fixes which triangles are lights and the light-choice distribution);
 * camera: origin, right, up, forward (12 floats).  out_image (w * h * 3) is
 * the rendered image; with dl_dimage (w * h * 3) the gradients of the loss
 * are added to d_albedo / d_emission (tri_count * 3, either may be NULL).
 * Returns 0, or -1 on a bad index. */
int orc_pt64(const float* verts, uint32_t vert_count, const uint32_t* tris, uint32_t tri_count,
    const float* albedo, const float* emission, const float* light_power_emission,
    const float* camera, float fov, uint32_t width, uint32_t height, uint32_t spp,
    uint32_t min_depth, uint32_t max_depth, uint64_t seed, uint32_t no_roulette,
    const float* dl_dimage, double* out_image, double* d_albedo, double* d_emission,
    uint64_t* out_rays);

#ifdef __cplusplus
}
#endif
#endif
