/* Float64 restatement of the "pt" estimator and of its gradient with
 * respect to per-triangle Lambert albedo and per-triangle emitted radiance.
 *
 * TEST INFRASTRUCTURE ONLY: the CPU reference for the GPU adjoint
 * (dort_gpu_adjoint_forward / _backward); the product library never links
 * it.
 *
 * Scope: the adjoint workload's scenes -- triangles with a Lambert material
 * whose albedo is given per triangle (0 = no BSDF), one-sided triangle
 * emitters (DiffuseLight on a triangle), a pinhole camera, the box filter,
 * min / max depth, MIS direct lighting, Russian roulette (optional).  Every
 * step follows the reference's PathRenderer:
 *   film position: pixel centre at sample 0, else jittered
 *                  (path_renderer.cpp:15-20)
 *   camera ray:    PinholeCamera::sample_ray_importance
 *                  (pinhole_camera.cpp:13-31; fov clamped, lua_camera.cpp:63-64)
 *   path loop:     PathRenderer::sample (path_renderer.cpp:23-111): emission
 *                  at bounce 0, direct lighting at bounces >= min_depth, BSDF
 *                  continuation, roulette after bounce 2 with
 *                  p = clamp(avg(f cos / pdf), 0.1, 0.99)
 *   direct light:  one light picked by power (scene.cpp:20-28,
 *                  discrete_distrib_1d.cpp:22-41), estimate_direct with the
 *                  balance heuristic over the BSDF and light strategies
 *                  (path_renderer.cpp:135-206)
 *   light:         Triangle::sample_point + Shape::sample_point_pivot /
 *                  point_pivot_pdf (triangle.cpp:62-80, shape.cpp:4-26),
 *                  DiffuseLight::eval_radiance one-sided
 *                  (diffuse_light.cpp:85-94); shadow segment ends 1e-3 short
 *                  of the light point (light.cpp:40-49)
 *   Lambert:       albedo / pi, cosine-hemisphere sampling on the side of wo
 *                  (lambert_material.cpp:5-35, monte_carlo.cpp:39-54)
 *   surface:       p from barycentrics, n = normalize(e2 x e1), frame
 *                  s = e1 / |e1|, ray epsilon |1e-3 t| (triangle.cpp:82-173)
 *   film:          non-finite or negative samples dropped, pixel = sum / count
 *                  (renderer.cpp:36-41, film.cpp:90-108)
 * Geometry and arithmetic are double; intersection is Moller-Trumbore over
 * every triangle (no BVH), closest hit with the larger index winning exact
 * ties (the device's order-independent rule).
 *
 * Random numbers: the device's counter-based streams, Philox4x32-10 (Salmon,
 * Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3", SC 2011)
 * keyed by the 64-bit seed with counter (pixel, sample, block, 0x64307274),
 * 24-bit uniforms; block 0 = camera jitter, block 1 + 3 b + {0, 1, 2} =
 * bounce b (light pick, BSDF-strategy sample, light sample, continuation,
 * roulette).  With the same numbers the restatement traces the same paths as
 * the GPU except where float and double rounding disagree (a ray grazing a
 * triangle edge, a uniform on a decision boundary).
 *
 * Gradient: every term a sample adds is a product of the albedos of the
 * Lambert vertices before it (the vertex that lights it included) and of one
 * light's radiance; roulette probabilities, light choice and MIS weights are
 * held fixed.  So dTerm / d albedo_v = Term / albedo_v for each such vertex
 * and dTerm / dLe = Term / Le (emission seen directly: the throughput).  Each
 * term's derivatives are added directly (forward mode per term), not by the
 * device's path replay, so the two formulations check each other.  A pixel's
 * samples are weighted by dLoss/dI(pixel) / (kept samples of the pixel).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double x, y, z; } d3;

static d3 D3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static d3 add(d3 a, d3 b) { return D3(a.x + b.x, a.y + b.y, a.z + b.z); }
static d3 sub(d3 a, d3 b) { return D3(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 scl(d3 a, double s) { return D3(a.x * s, a.y * s, a.z * s); }
static d3 mulv(d3 a, d3 b) { return D3(a.x * b.x, a.y * b.y, a.z * b.z); }
static double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static d3 cross(d3 a, d3 b) {
  return D3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double len(d3 a) { return sqrt(dot(a, a)); }
static d3 nrm(d3 a) { return scl(a, 1.0 / len(a)); }
static int black(d3 a) { return a.x == 0.0 && a.y == 0.0 && a.z == 0.0; }
static d3 ld3(const float* p) { return D3(p[0], p[1], p[2]); }

/* ---- Philox4x32-10 ---------------------------------------------------------- */

static void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for(int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static void rand4(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t block, double u[4]) {
  uint32_t c[4] = {pixel, sample, block, 0x64307274u};
  philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  for(int k = 0; k < 4; ++k) { u[k] = (double)(c[k] >> 8) * (1.0 / 16777216.0); }
}

/* ---- scene ------------------------------------------------------------------- */

typedef struct {
  uint32_t nt;
  d3 *p0, *e1, *e2, *n;       /* per triangle; n = normalize(e2 x e1) */
  double* area;
  const float* albedo;        /* nt * 3 */
  const float* emission;      /* nt * 3 (radiance in effect) */
  uint32_t nl;
  uint32_t* light_tri;
  int32_t* tri_light;         /* light index of a triangle, -1 if none */
  double* cdf;                /* nl + 1 */
} Scene64;

/* Moller-Trumbore (triangle.cpp:109-134) in double. */
static int mt(const Scene64* s, uint32_t k, d3 o, d3 d, double tmin, double tmax, double* t,
              double* b1o, double* b2o) {
  d3 e1 = s->e1[k], e2 = s->e2[k];
  d3 s1 = cross(d, e2);
  double det = dot(s1, e1);
  if(det == 0.0) { return 0; }
  double inv = 1.0 / det;
  d3 sv = sub(o, s->p0[k]);
  double b1 = inv * dot(s1, sv);
  if(b1 < 0.0 || b1 > 1.0) { return 0; }
  d3 s2 = cross(sv, e1);
  double b2 = inv * dot(s2, d);
  if(b2 < 0.0 || b1 + b2 > 1.0) { return 0; }
  double tt = inv * dot(s2, e2);
  if(tt < tmin || tt > tmax) { return 0; }
  *t = tt;
  *b1o = b1;
  *b2o = b2;
  return 1;
}

static int64_t closest(const Scene64* s, d3 o, double tmin, d3 d, double* t, double* b1,
                       double* b2, uint64_t* rays) {
  int64_t best = -1;
  double bt = INFINITY;
  *rays += 1;
  for(uint32_t k = 0; k < s->nt; ++k) {
    double tt, u, v;
    if(mt(s, k, o, d, tmin, bt, &tt, &u, &v) && (best < 0 || tt < bt || (int64_t)k > best)) {
      best = k;
      bt = tt;
      *b1 = u;
      *b2 = v;
    }
  }
  *t = bt;
  return best;
}

static int occluded(const Scene64* s, d3 o, double tmin, d3 d, double tmax, uint64_t* rays) {
  *rays += 1;
  for(uint32_t k = 0; k < s->nt; ++k) {
    double tt, u, v;
    if(mt(s, k, o, d, tmin, tmax, &tt, &u, &v)) { return 1; }
  }
  return 0;
}

/* DiscreteDistrib1d::sample (discrete_distrib_1d.cpp:22-36) */
static uint32_t distrib_sample(const double* cdf, uint32_t n, double u) {
  uint32_t begin = 0, end = n;
  while(begin + 1 < end) {
    uint32_t mid = begin + (end - begin) / 2;
    if(cdf[mid] < u) { begin = mid; } else { end = mid; }
  }
  return begin;
}

/* Shape::point_pivot_pdf on a light triangle (shape.cpp:15-26) */
static double light_pivot_pdf(const Scene64* s, uint32_t tri, d3 wi, d3 pivot) {
  d3 w = nrm(wi);
  double t, b1, b2;
  if(!mt(s, tri, pivot, w, 0.0, INFINITY, &t, &b1, &b2)) { return 0.0; }
  d3 pt = add(pivot, scl(w, t));
  d3 to = sub(pt, pivot);
  return (1.0 / s->area[tri]) * dot(to, to) / fabs(dot(w, s->n[tri]));
}

static d3 albedo_of(const Scene64* s, uint32_t tri) { return ld3(s->albedo + 3 * (size_t)tri); }
static d3 emission_of(const Scene64* s, uint32_t tri) {
  return ld3(s->emission + 3 * (size_t)tri);
}

/* ---- one sample ---------------------------------------------------------------- */

typedef struct {
  uint32_t w, h, spp, min_depth, max_depth, no_roulette;
  uint64_t seed;
  d3 origin, right, up, forward;
  double proj;
} Params64;

/* The terms of one sample: value and its contributors (for the gradient). */
typedef struct {
  d3 value;
  uint32_t nv;               /* Lambert vertices before it */
  uint32_t verts[64];
  int32_t light_tri;         /* the light whose radiance it carries, -1 none */
} Term;

typedef struct {
  Term* terms;
  uint32_t count, cap;
} Terms;

static void push_term(Terms* ts, d3 v, const uint32_t* verts, uint32_t nv, int32_t light_tri) {
  if(ts->count == ts->cap) {
    ts->cap = ts->cap ? 2 * ts->cap : 16;
    ts->terms = (Term*)realloc(ts->terms, ts->cap * sizeof(Term));
  }
  Term* t = &ts->terms[ts->count++];
  t->value = v;
  t->nv = nv;
  memcpy(t->verts, verts, nv * sizeof(uint32_t));
  t->light_tri = light_tri;
}

static void to_local(d3 s_, d3 t_, d3 n_, d3 v, d3* out) {
  *out = D3(dot(s_, v), dot(t_, v), dot(n_, v));
}

static d3 sample_path(const Scene64* sc, const Params64* pp, uint32_t pixel, uint32_t sample,
                      Terms* ts, uint64_t* rays) {
  uint32_t x = pixel % pp->w, y = pixel / pp->w;
  double fx, fy, u[4];
  if(sample == 0) {
    fx = x + 0.5;
    fy = y + 0.5;
  } else {
    rand4(pp->seed, pixel, sample, 0, u);
    fx = x + u[0];
    fy = y + u[1];
  }
  /* PinholeCamera::sample_ray_importance (pinhole_camera.cpp:13-31) */
  double W = pp->w, H = pp->h;
  double cx = fx / W - 0.5, cy = fy / H - 0.5, nx, ny;
  if(W > H) { nx = cx; ny = cy * H / W; } else { nx = cx * W / H; ny = cy; }
  d3 d = nrm(add(add(scl(pp->right, nx * pp->proj), scl(pp->up, ny * pp->proj)), pp->forward));
  d3 o = pp->origin;
  double tmin = 0.0;
  d3 sum = D3(0, 0, 0), thr = D3(1, 1, 1);
  uint32_t bounces = 0, verts[64], nv = 0;
  ts->count = 0;
  for(;;) {
    double t, b1, b2;
    int64_t hit = closest(sc, o, tmin, d, &t, &b1, &b2, rays);
    d3 p = D3(0, 0, 0), n = D3(0, 0, 1), fs = D3(1, 0, 0), ft = D3(0, 1, 0);
    double eps = 0.0;
    if(hit >= 0) {
      uint32_t k = (uint32_t)hit;
      p = add(sc->p0[k], add(scl(sc->e1[k], b1), scl(sc->e2[k], b2)));
      n = sc->n[k];
      eps = fabs(1e-3 * t);
      double l1 = len(sc->e1[k]);
      if(l1 >= 1e-9) {
        fs = scl(sc->e1[k], 1.0 / l1);
        ft = cross(n, fs);
      } else {
        /* coordinate_system (geometry.cpp:4-11) */
        fs = fabs(n.x) > fabs(n.y) ? nrm(D3(-n.z, 0, n.x)) : nrm(D3(0, -n.z, n.y));
        ft = cross(n, fs);
      }
    }
    /* emission seen at bounce 0 (path_renderer.cpp:42-57; Lambert has no
     * delta bounce) */
    if(bounces == 0 && bounces >= pp->min_depth && bounces <= pp->max_depth && hit >= 0 &&
       sc->tri_light[hit] >= 0 && dot(n, sub(o, p)) >= 0.0) {
      d3 c = mulv(thr, emission_of(sc, (uint32_t)hit));
      push_term(ts, c, verts, nv, (int32_t)hit);
      sum = add(sum, c);
    }
    bounces += 1;
    if(hit < 0 || bounces > pp->max_depth) { break; }
    uint32_t k = (uint32_t)hit;
    d3 alb = albedo_of(sc, k);
    int has_bsdf = !black(alb);
    d3 wo = nrm(scl(d, -1.0));
    d3 wo_l;
    to_local(fs, ft, n, wo, &wo_l);
    double r0[4], r1[4], r2[4];
    uint32_t blk = 1 + 3 * bounces;
    rand4(pp->seed, pixel, sample, blk, r0);
    rand4(pp->seed, pixel, sample, blk + 1, r1);
    rand4(pp->seed, pixel, sample, blk + 2, r2);
    if(has_bsdf) { verts[nv++] = k; }
    d3 f = scl(alb, 1.0 / M_PI);
    if(bounces >= pp->min_depth && has_bsdf && sc->nl > 0) {
      uint32_t li = distrib_sample(sc->cdf, sc->nl, r0[0]);
      double lpdf = sc->cdf[li + 1] - sc->cdf[li];
      uint32_t lt = sc->light_tri[li];
      if(lpdf != 0.0) {
        /* BSDF strategy (path_renderer.cpp:141-166) */
        double rr = sqrt(r0[1]), ph = 2.0 * M_PI * r0[2];
        double lx = cos(ph) * rr, ly = sin(ph) * rr;
        double lz = sqrt(fmax(0.0, 1.0 - lx * lx - ly * ly));
        lz = copysign(lz, wo_l.z);
        d3 wb = add(add(scl(fs, lx), scl(ft, ly)), scl(n, lz));
        double bpdf = fabs(lz) / M_PI;
        double dn = fabs(dot(n, wb));
        if(bpdf != 0.0 && dn * dn != 0.0) {
          double tt, c1, c2;
          int64_t h2 = closest(sc, p, eps, wb, &tt, &c1, &c2, rays);
          if(h2 == (int64_t)lt) {
            d3 ph2 = add(sc->p0[lt], add(scl(sc->e1[lt], c1), scl(sc->e2[lt], c2)));
            if(dot(sc->n[lt], sub(p, ph2)) >= 0.0) {
              double lp = light_pivot_pdf(sc, lt, wb, p);
              double wgt = bpdf / (bpdf + lp);
              d3 c = scl(mulv(mulv(f, emission_of(sc, lt)), thr), wgt * dn / bpdf / lpdf);
              push_term(ts, c, verts, nv, (int32_t)lt);
              sum = add(sum, c);
            }
          }
        }
        /* light strategy (path_renderer.cpp:168-206) */
        double sr = sqrt(r1[0]);
        double lb1 = 1.0 - sr, lb2 = r1[1] * sr;
        d3 pt = add(sc->p0[lt], add(scl(sc->e1[lt], lb1), scl(sc->e2[lt], lb2)));
        d3 to = sub(p, pt);
        double lspdf = (1.0 / sc->area[lt]) * dot(to, to) / fabs(dot(sc->n[lt], nrm(to)));
        d3 wi = nrm(sub(pt, p));
        if(lspdf != 0.0 && dot(wi, sc->n[lt]) < 0.0) {
          d3 wi_l;
          to_local(fs, ft, n, wi, &wi_l);
          double dn2 = fabs(dot(n, wi));
          if(wo_l.z * wi_l.z > 0.0 && dn2 * dn2 != 0.0) {
            double dist = len(sub(pt, p));
            if(!occluded(sc, p, eps, scl(sub(pt, p), 1.0 / dist), dist - 1e-3, rays)) {
              double bp = fabs(wi_l.z) / M_PI;
              double wgt = lspdf / (lspdf + bp);
              d3 c = scl(mulv(mulv(f, emission_of(sc, lt)), thr), wgt * dn2 / lspdf / lpdf);
              push_term(ts, c, verts, nv, (int32_t)lt);
              sum = add(sum, c);
            }
          }
        }
      }
    }
    /* continuation (path_renderer.cpp:82-106) */
    if(!has_bsdf || bounces == pp->max_depth) { break; }
    double rr = sqrt(r1[2]), ph = 2.0 * M_PI * r1[3];
    double cx2 = cos(ph) * rr, cy2 = sin(ph) * rr;
    double cz = sqrt(fmax(0.0, 1.0 - cx2 * cx2 - cy2 * cy2));
    cz = copysign(cz, wo_l.z);
    d3 wn = add(add(scl(fs, cx2), scl(ft, cy2)), scl(n, cz));
    double cpdf = fabs(cz) / M_PI;
    double dn3 = fabs(dot(n, wn));
    if(cpdf == 0.0 || dn3 * dn3 == 0.0) { break; }
    d3 contrib = scl(f, dn3 / cpdf);
    thr = mulv(thr, contrib);
    if(bounces >= 2 && bounces > pp->min_depth && !pp->no_roulette) {
      double survive = (contrib.x + contrib.y + contrib.z) / 3.0;
      survive = survive < 0.1 ? 0.1 : (survive > 0.99 ? 0.99 : survive);
      if(r2[1] > survive) { break; }
      thr = scl(thr, 1.0 / survive);
    }
    o = p;
    d = wn;
    tmin = eps;
  }
  return sum;
}

static int kept(d3 L) {
  return isfinite(L.x) && isfinite(L.y) && isfinite(L.z) && L.x >= 0 && L.y >= 0 && L.z >= 0;
}

int orc_pt64(const float* verts, uint32_t vert_count, const uint32_t* tris, uint32_t tri_count,
             const float* albedo, const float* emission, const float* light_power_emission,
             const float* camera, float fov, uint32_t width, uint32_t height, uint32_t spp,
             uint32_t min_depth, uint32_t max_depth, uint64_t seed, uint32_t no_roulette,
             const float* dl_dimage, double* out_image, double* d_albedo, double* d_emission,
             uint64_t* out_rays) {
  Scene64 sc;
  memset(&sc, 0, sizeof(sc));
  sc.nt = tri_count;
  sc.p0 = (d3*)malloc(sizeof(d3) * tri_count);
  sc.e1 = (d3*)malloc(sizeof(d3) * tri_count);
  sc.e2 = (d3*)malloc(sizeof(d3) * tri_count);
  sc.n = (d3*)malloc(sizeof(d3) * tri_count);
  sc.area = (double*)malloc(sizeof(double) * tri_count);
  sc.tri_light = (int32_t*)malloc(sizeof(int32_t) * tri_count);
  sc.light_tri = (uint32_t*)malloc(sizeof(uint32_t) * tri_count);
  sc.cdf = (double*)malloc(sizeof(double) * (tri_count + 1));
  sc.albedo = albedo;
  sc.emission = emission;
  double total = 0.0;
  for(uint32_t k = 0; k < tri_count; ++k) {
    for(int j = 0; j < 3; ++j) {
      if(tris[3 * k + j] >= vert_count) { return -1; }
    }
    d3 a = ld3(verts + 3 * (size_t)tris[3 * k]);
    d3 b = ld3(verts + 3 * (size_t)tris[3 * k + 1]);
    d3 c = ld3(verts + 3 * (size_t)tris[3 * k + 2]);
    sc.p0[k] = a;
    sc.e1[k] = sub(b, a);
    sc.e2[k] = sub(c, a);
    d3 cr = cross(sc.e2[k], sc.e1[k]);
    sc.area[k] = 0.5 * len(cr);
    sc.n[k] = len(cr) > 0 ? nrm(cr) : D3(0, 0, 1);
    sc.tri_light[k] = -1;
    const float* le = light_power_emission + 3 * (size_t)k;
    if(le[0] != 0.f || le[1] != 0.f || le[2] != 0.f) {
      /* scene.cpp:20-28: light choice by approximate power (area x mean Le) */
      sc.cdf[sc.nl] = total;
      total += sc.area[k] * (le[0] + le[1] + le[2]) / 3.0;
      sc.tri_light[k] = (int32_t)sc.nl;
      sc.light_tri[sc.nl++] = k;
    }
  }
  sc.cdf[sc.nl] = total;
  for(uint32_t l = 0; l <= sc.nl; ++l) { sc.cdf[l] = total > 0 ? sc.cdf[l] / total : 0.0; }

  Params64 pp;
  pp.w = width;
  pp.h = height;
  pp.spp = spp;
  pp.min_depth = min_depth;
  pp.max_depth = max_depth;
  pp.no_roulette = no_roulette;
  pp.seed = seed;
  pp.origin = ld3(camera);
  pp.right = ld3(camera + 3);
  pp.up = ld3(camera + 6);
  pp.forward = ld3(camera + 9);
  double fv = fov;
  if(!(fv >= 1e-2)) { fv = 1e-2; }
  if(fv > M_PI) { fv = M_PI; }
  pp.proj = 2.0 * tan(0.5 * fv);

  Terms ts = {0};
  uint64_t rays = 0;
  const uint32_t npix = width * height;
  d3* Ls = (d3*)malloc(sizeof(d3) * spp);
  for(uint32_t pixel = 0; pixel < npix; ++pixel) {
    d3 acc = D3(0, 0, 0);
    uint32_t count = 0;
    for(uint32_t s = 0; s < spp; ++s) {
      Ls[s] = sample_path(&sc, &pp, pixel, s, &ts, &rays);
      if(kept(Ls[s])) {
        acc = add(acc, Ls[s]);
        count += 1;
      }
    }
    if(out_image) {
      out_image[3 * (size_t)pixel] = count ? acc.x / count : 0.0;
      out_image[3 * (size_t)pixel + 1] = count ? acc.y / count : 0.0;
      out_image[3 * (size_t)pixel + 2] = count ? acc.z / count : 0.0;
    }
    if(!dl_dimage || !count) { continue; }
    d3 adj = scl(ld3(dl_dimage + 3 * (size_t)pixel), 1.0 / count);
    if(black(adj)) { continue; }
    for(uint32_t s = 0; s < spp; ++s) {
      if(!kept(Ls[s])) { continue; }
      sample_path(&sc, &pp, pixel, s, &ts, &rays);      /* the sample's terms again */
      for(uint32_t q = 0; q < ts.count; ++q) {
        const Term* t = &ts.terms[q];
        d3 g = mulv(adj, t->value);
        for(uint32_t v = 0; d_albedo && v < t->nv; ++v) {
          uint32_t tri = t->verts[v];
          d3 a = albedo_of(&sc, tri);
          double* o = d_albedo + 3 * (size_t)tri;
          if(a.x > 0) { o[0] += g.x / a.x; }
          if(a.y > 0) { o[1] += g.y / a.y; }
          if(a.z > 0) { o[2] += g.z / a.z; }
        }
        if(d_emission && t->light_tri >= 0) {
          d3 le = emission_of(&sc, (uint32_t)t->light_tri);
          double* o = d_emission + 3 * (size_t)t->light_tri;
          if(le.x > 0) { o[0] += g.x / le.x; }
          if(le.y > 0) { o[1] += g.y / le.y; }
          if(le.z > 0) { o[2] += g.z / le.z; }
        }
      }
    }
  }
  free(Ls);
  free(ts.terms);
  free(sc.p0); free(sc.e1); free(sc.e2); free(sc.n); free(sc.area);
  free(sc.tri_light); free(sc.light_tri); free(sc.cdf);
  if(out_rays) { *out_rays = rays; }
  return 0;
}
