/* CPU restatement of the reference's BVH build and traversal and of its
 * Moller-Trumbore ray/triangle test.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Every arithmetic step keeps the
 * reference's float operation order; the file is compiled with
 * -ffp-contract=off so that no multiply-add is fused, matching the reference
 * built for baseline x86-64 (SSE, no FMA).
 *
 * Reference files (paths inside the reference project):
 *   include/dort/bvh.hpp, src/dort/bvh.cpp      build + traversal
 *   include/dort/box.hpp, src/dort/box.cpp      Box, union, slab test
 *   src/dort/triangle.cpp                       Triangle::hit_p, TriangleUv::hit
 *   include/dort/math.hpp                       min/max/clamp/arg_max_3
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* ---- scalar helpers (math.hpp) ------------------------------------------ */

/* min/max exactly as math.hpp:63-64: the second operand wins only on a strict
 * comparison, which fixes the sign chosen for +0/-0. */
static inline float fmin_ref(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_ref(float a, float b) { return (a < b) ? b : a; }

/* floor_int32 (math.hpp:66) is int32_t(floor(a)); on x86-64 the conversion
 * of NaN or an out-of-range value yields INT32_MIN ("integer indefinite"). */
static inline int32_t floor_i32(float a) {
  float f = floorf(a);
  if(!(f >= -2147483648.f && f < 2147483648.f)) { return INT32_MIN; }
  return (int32_t)f;
}

/* arg_max_3 (math.hpp:116-122). */
static inline uint8_t arg_max_3(float a0, float a1, float a2) {
  uint32_t bit_0 = a0 < a1;
  uint32_t bit_1 = a0 < a2;
  uint32_t bit_2 = a1 < a2;
  static const uint8_t opts[8] = { 0, 1, 255, 1, 0, 255, 2, 2 };
  return opts[bit_0 | (bit_1 << 1) | (bit_2 << 2)];
}

/* ---- Box (box.hpp, box.cpp) --------------------------------------------- */

typedef struct { float lo[3]; float hi[3]; } box3;

static inline box3 box_empty(void) {   /* box.hpp:9-11 */
  box3 b = { { INFINITY, INFINITY, INFINITY }, { -INFINITY, -INFINITY, -INFINITY } };
  return b;
}

static inline box3 box_union(box3 a, box3 b) {   /* box.cpp:4-14 */
  box3 r;
  for(int i = 0; i < 3; ++i) {
    r.lo[i] = fmin_ref(a.lo[i], b.lo[i]);
    r.hi[i] = fmax_ref(a.hi[i], b.hi[i]);
  }
  return r;
}

static inline box3 box_union_pt(box3 a, const float* p) {   /* box.cpp:16-26 */
  box3 r;
  for(int i = 0; i < 3; ++i) {
    r.lo[i] = fmin_ref(a.lo[i], p[i]);
    r.hi[i] = fmax_ref(a.hi[i], p[i]);
  }
  return r;
}

static inline void box_centroid(const box3* b, float* c) {   /* box.hpp:32-34 */
  for(int i = 0; i < 3; ++i) { c[i] = (b->hi[i] + b->lo[i]) * 0.5f; }
}

/* Box::area (box.hpp:27-30), including the reference's missing x*y term. */
static inline float box_area(const box3* b) {
  float rx = b->hi[0] - b->lo[0];
  float ry = b->hi[1] - b->lo[1];
  float rz = b->hi[2] - b->lo[2];
  return 2.f * (ry * rz + rx * rz + ry * rz);
}

static inline uint8_t box_max_axis(const box3* b) {   /* box.hpp:40-42 */
  return arg_max_3(b->hi[0] - b->lo[0], b->hi[1] - b->lo[1], b->hi[2] - b->lo[2]);
}

/* Box::fast_hit_p (box.cpp:57-90). */
static inline int box_fast_hit_p(const box3* b, const float* o, const float* inv,
    const int* neg, float ray_tmin, float ray_tmax)
{
  const float* lo_hi[2] = { b->lo, b->hi };
  float t_min = (lo_hi[neg[0]][0] - o[0]) * inv[0];
  float t_max = (lo_hi[1 - neg[0]][0] - o[0]) * inv[0];
  float ty_min = (lo_hi[neg[1]][1] - o[1]) * inv[1];
  float ty_max = (lo_hi[1 - neg[1]][1] - o[1]) * inv[1];
  if(t_min > ty_max || ty_min > t_max) { return 0; }
  if(ty_min > t_min) { t_min = ty_min; }
  if(ty_max < t_max) { t_max = ty_max; }
  float tz_min = (lo_hi[neg[2]][2] - o[2]) * inv[2];
  float tz_max = (lo_hi[1 - neg[2]][2] - o[2]) * inv[2];
  if(t_min > tz_max || t_max < tz_min) { return 0; }
  if(tz_min > t_min) { t_min = tz_min; }
  if(t_max > tz_max) { t_max = tz_max; }
  return (t_min < ray_tmax) && (t_max > ray_tmin);
}

/* ---- Moller-Trumbore (triangle.cpp:14-46, 102-134) ---------------------- */

static inline float dot3(const float* a, const float* b) {   /* vec_3.hpp dot */
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static inline void cross3(const float* a, const float* b, float* r) {   /* vec_3.hpp cross */
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

/* Shared body of Triangle::hit_p and TriangleUv::hit; both run the same
 * arithmetic and the same rejection tests in the same order. */
static inline int mt_hit(const float* p0, const float* p1, const float* p2,
    const float* o, const float* d, float t_min, float t_max, float* out_tb)
{
  float e1[3] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
  float e2[3] = { p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2] };
  float s1[3];
  cross3(d, e2, s1);
  float det = dot3(s1, e1);
  if(det == 0.f) { return 0; }
  float inv_det = 1.f / det;

  float s[3] = { o[0] - p0[0], o[1] - p0[1], o[2] - p0[2] };
  float b1 = inv_det * dot3(s1, s);
  if(b1 < 0.f || b1 > 1.f) { return 0; }

  float s2[3];
  cross3(s, e1, s2);
  float b2 = inv_det * dot3(s2, d);
  if(b2 < 0.f || b1 + b2 > 1.f) { return 0; }

  float t = inv_det * dot3(s2, e2);
  if(t < t_min || t > t_max) { return 0; }
  out_tb[0] = t;
  out_tb[1] = b1;
  out_tb[2] = b2;
  return 1;
}

int orc_triangle_hit(const float* p0, const float* p1, const float* p2,
    const float* ray, float* out_tb)
{
  return mt_hit(p0, p1, p2, ray, ray + 4, ray[3], ray[7], out_tb);
}

/* ---- BVH build (bvh.cpp:9-416) ------------------------------------------ */

typedef struct {          /* Bvh::LinearNode (bvh.hpp:34-40) */
  box3 bounds;
  uint32_t offset_or_left;
  uint16_t count_or_zero;
  uint8_t axis;
} lnode;

typedef struct {          /* Bvh::ElementInfo (bvh.hpp:42-45) */
  uint32_t elem;
  box3 bounds;
} einfo;

typedef struct {          /* Bvh::NodeInfo (bvh.hpp:56-62) */
  box3 bounds;
  box3 centroid_bounds;
  uint32_t begin, end, linear_idx;
} ninfo;

typedef struct {          /* Bvh::SplitInfo (bvh.hpp:64-69) */
  box3 left_bounds, right_bounds;
  box3 left_centroid_bounds, right_centroid_bounds;
  uint32_t mid;
  int prefer_leaf;
} sinfo;

struct orc_bvh {
  const float* verts;       /* borrowed during build only */
  float* points;            /* owned copy, 3 floats per vertex */
  uint32_t* tri_idx;        /* owned copy, 3 per triangle */
  uint32_t tri_count;
  lnode* nodes;
  uint32_t node_count, node_cap;
  uint32_t* ordered_elems;  /* vertex-array offsets (3 * triangle) */
};

typedef struct {
  struct orc_bvh* bvh;
  einfo* infos;
  int split_method;
  uint32_t leaf_size, max_leaf_size;
  uint32_t free_idx;
} bctx;

static void tri_points(const struct orc_bvh* b, uint32_t elem,
    const float** p0, const float** p1, const float** p2)
{
  *p0 = b->points + 3 * (size_t)b->tri_idx[elem];
  *p1 = b->points + 3 * (size_t)b->tri_idx[elem + 1];
  *p2 = b->points + 3 * (size_t)b->tri_idx[elem + 2];
}

static void write_node(bctx* ctx, uint32_t idx, lnode n) {   /* bvh.cpp:178-199 */
  struct orc_bvh* b = ctx->bvh;
  if(idx >= b->node_cap) {
    uint32_t cap = b->node_cap ? b->node_cap : 16;
    while(cap <= idx) { cap *= 2; }
    b->nodes = (lnode*)realloc(b->nodes, sizeof(lnode) * cap);
    b->node_cap = cap;
  }
  b->nodes[idx] = n;
  if(idx + 1 > b->node_count) { b->node_count = idx + 1; }
}

static inline float info_centroid_axis(const einfo* e, uint8_t axis) {
  float c[3];
  box_centroid(&e->bounds, c);
  return c[axis];
}

/* std::partition as libstdc++ implements it for random-access ranges (the
 * two-ended swap scan); the element order it leaves decides the order of
 * triangles inside leaves.  Predicate: bvh.cpp:392-397. */
static uint32_t partition(bctx* ctx, uint32_t begin, uint32_t end,
    uint8_t axis, float separator)
{
  einfo* first = ctx->infos + begin;
  einfo* last = ctx->infos + end;
  for(;;) {
    for(;;) {
      if(first == last) { return (uint32_t)(first - ctx->infos); }
      if(info_centroid_axis(first, axis) < separator) { ++first; } else { break; }
    }
    --last;
    for(;;) {
      if(first == last) { return (uint32_t)(first - ctx->infos); }
      if(!(info_centroid_axis(last, axis) < separator)) { --last; } else { break; }
    }
    einfo tmp = *first; *first = *last; *last = tmp;
    ++first;
  }
}

/* Bvh::split_middle (bvh.cpp:201-278). */
static sinfo split_middle(bctx* ctx, const ninfo* node, uint8_t axis) {
  uint32_t begin = node->begin, end = node->end;
  float c[3];
  box_centroid(&node->centroid_bounds, c);
  uint32_t mid = partition(ctx, begin, end, axis, c[axis]);
  if(mid == begin || mid + 1 == end) { mid = begin + (end - begin) / 2; }

  sinfo s;
  s.left_bounds = box_empty(); s.left_centroid_bounds = box_empty();
  s.right_bounds = box_empty(); s.right_centroid_bounds = box_empty();
  for(uint32_t i = begin; i < mid; ++i) {
    float ce[3];
    box_centroid(&ctx->infos[i].bounds, ce);
    s.left_bounds = box_union(s.left_bounds, ctx->infos[i].bounds);
    s.left_centroid_bounds = box_union_pt(s.left_centroid_bounds, ce);
  }
  for(uint32_t i = mid; i < end; ++i) {
    float ce[3];
    box_centroid(&ctx->infos[i].bounds, ce);
    s.right_bounds = box_union(s.right_bounds, ctx->infos[i].bounds);
    s.right_centroid_bounds = box_union_pt(s.right_centroid_bounds, ce);
  }
  s.mid = mid;
  s.prefer_leaf = 0;
  return s;
}

typedef struct {          /* Bvh::BucketInfo (bvh.hpp:47-54) */
  uint32_t count;
  box3 bounds, centroid_bounds, prefix_bounds, postfix_bounds;
  uint32_t prefix_count;
} bucket;

/* Bvh::sah_split_cost (bvh.cpp:401-416): SAH_TRAVERSAL_COST = 1,
 * SAH_INTERSECTION_COST = 2 (bvh.hpp:31-32). */
static int32_t sah_split_cost(const box3* centroid_bounds, const bucket* bk,
    uint32_t elem_count)
{
  uint32_t count_l = bk->prefix_count;
  uint32_t count_r = elem_count - count_l;
  if(count_l == 0 || count_r == 0) { return INT32_MAX; }
  float area_l = box_area(&bk->prefix_bounds);
  float area_r = box_area(&bk->postfix_bounds);
  float isects = (area_l * (float)count_l + area_r * (float)count_r)
    / box_area(centroid_bounds);
  /* 1 + INT32_MIN cannot overflow; other values are small. */
  return (int32_t)((int64_t)1 + floor_i32(isects * 2.f));
}

#define SAH_BUCKETS 12    /* BvhOpts::sah_bucket_count (bvh.hpp:20) */

/* Bvh::split_sah (bvh.cpp:280-383). */
static sinfo split_sah(bctx* ctx, const ninfo* node, uint8_t axis) {
  float extent = node->centroid_bounds.hi[axis] - node->centroid_bounds.lo[axis];
  float bounds_min = node->centroid_bounds.lo[axis];
  float inv_extent = 1.f / extent;
  uint32_t begin = node->begin, end = node->end;

  bucket bk[SAH_BUCKETS];
  for(int b = 0; b < SAH_BUCKETS; ++b) {
    bk[b].count = 0;
    bk[b].bounds = box_empty();
    bk[b].centroid_bounds = box_empty();
    bk[b].prefix_bounds = box_empty();
    bk[b].postfix_bounds = box_empty();
    bk[b].prefix_count = 0;
  }

  for(uint32_t i = begin; i < end; ++i) {
    const einfo* e = &ctx->infos[i];
    float ce[3];
    box_centroid(&e->bounds, ce);
    float elem_pos = ce[axis] - bounds_min;
    /* clamp(uint32_t(floor_int32(12 * pos * inv_extent)), 0, 11) */
    uint32_t idx = (uint32_t)floor_i32((float)SAH_BUCKETS * elem_pos * inv_extent);
    if(idx > SAH_BUCKETS - 1) { idx = SAH_BUCKETS - 1; }
    bk[idx].count += 1;
    bk[idx].bounds = box_union(bk[idx].bounds, e->bounds);
    bk[idx].centroid_bounds = box_union_pt(bk[idx].centroid_bounds, ce);
  }

  box3 prefix = box_empty();
  uint32_t prefix_count = 0;
  for(int b = 0; b < SAH_BUCKETS; ++b) {
    prefix = box_union(prefix, bk[b].bounds);
    prefix_count += bk[b].count;
    bk[b].prefix_bounds = prefix;
    bk[b].prefix_count = prefix_count;
  }
  box3 postfix = box_empty();
  for(int b = SAH_BUCKETS; b-- > 0; ) {
    bk[b].postfix_bounds = postfix;
    postfix = box_union(postfix, bk[b].bounds);
  }

  int32_t best_cost = sah_split_cost(&node->centroid_bounds, &bk[0], end - begin);
  uint32_t best_bucket = 0;
  for(uint32_t b = 1; b < SAH_BUCKETS - 1; ++b) {
    int32_t cost = sah_split_cost(&node->centroid_bounds, &bk[b], end - begin);
    if(cost < best_cost) { best_cost = cost; best_bucket = b; }
  }

  int32_t leaf_cost = 2 * (int32_t)(end - begin);
  float separator = (float)(best_bucket + 1) / (float)SAH_BUCKETS * extent + bounds_min;

  sinfo s;
  s.prefer_leaf = leaf_cost < best_cost;
  s.mid = partition(ctx, begin, end, axis, separator);
  s.left_bounds = box_empty(); s.left_centroid_bounds = box_empty();
  s.right_bounds = box_empty(); s.right_centroid_bounds = box_empty();
  for(uint32_t b = 0; b < SAH_BUCKETS; ++b) {
    if(b <= best_bucket) {
      s.left_bounds = box_union(s.left_bounds, bk[b].bounds);
      s.left_centroid_bounds = box_union(s.left_centroid_bounds, bk[b].centroid_bounds);
    } else {
      s.right_bounds = box_union(s.right_bounds, bk[b].bounds);
      s.right_centroid_bounds = box_union(s.right_centroid_bounds, bk[b].centroid_bounds);
    }
  }
  if(s.mid == begin || s.mid + 1 == end) {
    s.mid = begin + (end - begin) / 2;
    s.left_bounds = s.right_bounds = node->bounds;
    s.left_centroid_bounds = s.right_centroid_bounds = node->centroid_bounds;
  }
  return s;
}

/* Bvh::build_node (bvh.cpp:98-176), serial.  The reference builds large
 * nodes with a thread pool, but every parallel step there is a union or a
 * count (order-independent) and the recursion order only changes the linear
 * node indices, not the tree, so the serial build yields the same tree. */
static void build_node(bctx* ctx, const ninfo* node) {
  /* Explicit stack instead of recursion: big degenerate meshes can go deep. */
  size_t cap = 64, top = 0;
  ninfo* stack = (ninfo*)malloc(sizeof(ninfo) * cap);
  stack[top++] = *node;
  while(top > 0) {
    ninfo n = stack[--top];
    uint32_t elem_count = n.end - n.begin;
    uint8_t axis = box_max_axis(&n.centroid_bounds);
    int make_leaf = elem_count <= ctx->leaf_size;
    sinfo split;
    memset(&split, 0, sizeof(split));
    if(!make_leaf) {
      split = ctx->split_method == 1 ? split_sah(ctx, &n, axis)
                                     : split_middle(ctx, &n, axis);
      make_leaf = split.prefer_leaf && elem_count <= ctx->max_leaf_size;
    }
    if(make_leaf) {
      for(uint32_t i = n.begin; i < n.end; ++i) {
        ctx->bvh->ordered_elems[i] = ctx->infos[i].elem;
      }
      lnode leaf = { n.bounds, n.begin, (uint16_t)elem_count, axis };
      write_node(ctx, n.linear_idx, leaf);
    } else {
      ninfo left, right;
      left.bounds = split.left_bounds;
      left.centroid_bounds = split.left_centroid_bounds;
      left.begin = n.begin; left.end = split.mid;
      left.linear_idx = ctx->free_idx; ctx->free_idx += 2;
      right.bounds = split.right_bounds;
      right.centroid_bounds = split.right_centroid_bounds;
      right.begin = split.mid; right.end = n.end;
      right.linear_idx = left.linear_idx + 1;
      lnode branch = { n.bounds, left.linear_idx, 0, axis };
      write_node(ctx, n.linear_idx, branch);
      if(top + 2 > cap) { cap *= 2; stack = (ninfo*)realloc(stack, sizeof(ninfo) * cap); }
      stack[top++] = right;   /* left is built first, as in the reference */
      stack[top++] = left;
    }
  }
  free(stack);
}

orc_bvh* orc_bvh_build(const float* verts, uint32_t vert_count,
    const uint32_t* tri_idx, uint32_t tri_count, int split_method,
    uint32_t leaf_size, uint32_t max_leaf_size)
{
  struct orc_bvh* b = (struct orc_bvh*)calloc(1, sizeof(*b));
  b->points = (float*)malloc(sizeof(float) * 3 * (size_t)(vert_count ? vert_count : 1));
  memcpy(b->points, verts, sizeof(float) * 3 * (size_t)vert_count);
  b->tri_idx = (uint32_t*)malloc(sizeof(uint32_t) * 3 * (size_t)(tri_count ? tri_count : 1));
  memcpy(b->tri_idx, tri_idx, sizeof(uint32_t) * 3 * (size_t)tri_count);
  b->tri_count = tri_count;
  b->ordered_elems = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(tri_count ? tri_count : 1));

  bctx ctx;
  ctx.bvh = b;
  ctx.split_method = split_method;
  /* bvh.cpp:26-27 */
  ctx.max_leaf_size = max_leaf_size < 0xffffu ? max_leaf_size : 0xffffu;
  ctx.leaf_size = leaf_size < ctx.max_leaf_size ? leaf_size : ctx.max_leaf_size;
  ctx.free_idx = 1;
  ctx.infos = (einfo*)malloc(sizeof(einfo) * (size_t)(tri_count ? tri_count : 1));

  /* Bvh::compute_build_infos (bvh.cpp:57-96). */
  box3 root_bounds = box_empty();
  box3 root_centroid_bounds = box_empty();
  for(uint32_t i = 0; i < tri_count; ++i) {
    const float *p0, *p1, *p2;
    tri_points(b, 3 * i, &p0, &p1, &p2);
    box3 eb = box_empty();                 /* Triangle::bounds, triangle.cpp:48-54 */
    eb = box_union_pt(eb, p0);
    eb = box_union_pt(eb, p1);
    eb = box_union_pt(eb, p2);
    ctx.infos[i].elem = 3 * i;
    ctx.infos[i].bounds = eb;
    root_bounds = box_union(root_bounds, eb);
  }
  /* bvh.cpp:92 unions the element bounds (not the centroids) into the root
   * centroid bounds; the restatement keeps that. */
  root_centroid_bounds = box_union(root_centroid_bounds, root_bounds);

  ninfo root = { root_bounds, root_centroid_bounds, 0, tri_count, 0 };
  build_node(&ctx, &root);
  free(ctx.infos);
  return b;
}

void orc_bvh_free(orc_bvh* b) {
  if(!b) { return; }
  free(b->points); free(b->tri_idx); free(b->nodes); free(b->ordered_elems);
  free(b);
}

uint32_t orc_bvh_node_count(const orc_bvh* b) { return b->node_count; }

static void dump_rec(const struct orc_bvh* b, uint32_t idx, float* boxes,
    uint32_t* meta, uint32_t* out)
{
  const lnode* n = &b->nodes[idx];
  uint32_t k = (*out)++;
  memcpy(boxes + 6 * (size_t)k, n->bounds.lo, 3 * sizeof(float));
  memcpy(boxes + 6 * (size_t)k + 3, n->bounds.hi, 3 * sizeof(float));
  meta[3 * (size_t)k] = n->count_or_zero ? n->offset_or_left : 0;
  meta[3 * (size_t)k + 1] = n->count_or_zero;
  meta[3 * (size_t)k + 2] = n->axis;
  if(n->count_or_zero == 0 && b->tri_count > 0) {
    dump_rec(b, n->offset_or_left, boxes, meta, out);
    dump_rec(b, n->offset_or_left + 1, boxes, meta, out);
  }
}

void orc_bvh_nodes(const orc_bvh* b, float* boxes, uint32_t* meta) {
  uint32_t out = 0;
  if(b->node_count > 0) { dump_rec(b, 0, boxes, meta, &out); }
}

/* ---- Traversal (bvh.cpp:418-469 + mesh_bvh_primitive.cpp:13-45) -------- */

void orc_raycast(const orc_bvh* b, const float* rays, uint64_t ray_count,
    int any_hit, uint32_t* out_prim, float* out_tb,
    uint32_t* out_nodes, uint32_t* out_tests)
{
  for(uint64_t r = 0; r < ray_count; ++r) {
    const float* ray = rays + 8 * r;
    const float* o = ray;
    const float* d = ray + 4;
    float t_min = ray[3];
    float t_max = ray[7];
    float inv[3] = { 1.f / d[0], 1.f / d[1], 1.f / d[2] };
    int neg[3] = { d[0] < 0.f, d[1] < 0.f, d[2] < 0.f };

    uint32_t stack[64];
    uint32_t top = 0, idx = 0, visited = 0, tests = 0;
    int found = 0;
    uint32_t hit_elem = 0;
    float hit_tb[3] = { 0.f, 0.f, 0.f };

    if(b->tri_count > 0) {
      for(;;) {
        const lnode* n = &b->nodes[idx];
        visited += 1;
        int stop = 0;
        if(box_fast_hit_p(&n->bounds, o, inv, neg, t_min, t_max)) {
          if(n->count_or_zero == 0) {
            uint32_t left = n->offset_or_left, right = left + 1;
            if(neg[n->axis]) { stack[top++] = left; idx = right; }
            else { stack[top++] = right; idx = left; }
            continue;
          }
          for(uint32_t i = 0; i < n->count_or_zero; ++i) {
            uint32_t elem = b->ordered_elems[n->offset_or_left + i];
            const float *p0, *p1, *p2;
            tri_points(b, elem, &p0, &p1, &p2);
            float tb[3];
            tests += 1;
            if(mt_hit(p0, p1, p2, o, d, t_min, t_max, tb)) {
              found = 1;
              if(any_hit) { stop = 1; break; }
              t_max = tb[0];         /* mesh_bvh_primitive.cpp:20 */
              hit_elem = elem;
              hit_tb[0] = tb[0]; hit_tb[1] = tb[1]; hit_tb[2] = tb[2];
            }
          }
        }
        if(stop || top == 0) { break; }
        idx = stack[--top];
      }
    }

    if(any_hit) {
      out_prim[r] = found ? 1u : 0u;
    } else if(found) {
      out_prim[r] = hit_elem / 3;
      out_tb[3 * r] = hit_tb[0];
      out_tb[3 * r + 1] = hit_tb[1];
      out_tb[3 * r + 2] = hit_tb[2];
    } else {
      out_prim[r] = 0xffffffffu;
    }
    if(out_nodes) { out_nodes[r] = visited; }
    if(out_tests) { out_tests[r] = tests; }
  }
}

void orc_raycast_brute(const float* verts, const uint32_t* tri_idx,
    uint32_t tri_count, const float* rays, uint64_t ray_count,
    uint32_t* out_prim, float* out_tb)
{
  for(uint64_t r = 0; r < ray_count; ++r) {
    const float* ray = rays + 8 * r;
    float t_max = ray[7];
    uint32_t best = 0xffffffffu;
    float best_tb[3] = { 0.f, 0.f, 0.f };
    for(uint32_t i = 0; i < tri_count; ++i) {
      float tb[3];
      if(mt_hit(verts + 3 * (size_t)tri_idx[3 * i], verts + 3 * (size_t)tri_idx[3 * i + 1],
            verts + 3 * (size_t)tri_idx[3 * i + 2], ray, ray + 4, ray[3], t_max, tb)) {
        /* strictly nearer wins; equal t keeps the larger index (a fixed,
         * order-independent tie rule for classification) */
        if(best == 0xffffffffu || tb[0] < best_tb[0] || i > best) {
          best = i;
          best_tb[0] = tb[0]; best_tb[1] = tb[1]; best_tb[2] = tb[2];
          t_max = tb[0];
        }
      }
    }
    out_prim[r] = best;
    if(best != 0xffffffffu) {
      out_tb[3 * r] = best_tb[0]; out_tb[3 * r + 1] = best_tb[1]; out_tb[3 * r + 2] = best_tb[2];
    }
  }
}
