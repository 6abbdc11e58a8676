// The per-node steps of turning a binary BVH into the wide format of
// bvh_build.h, shared by the host builder (bvh_build.cpp) and the device
// builder (bvh_device.cu) so that both make bit-identical wide nodes from the
// same binary tree:
//
//   open_candidates   up to `width` children: the binary node's two children,
//                     then repeatedly the candidate of largest surface area
//                     that is not a binary leaf replaced by its children
//   assign_slots      greedy octant assignment: each (candidate, slot) pair
//                     is scored by how far the candidate's centre lies in the
//                     slot's octant direction from the node's centre; the
//                     lowest score is taken first
//   quantize_axis     8-bit conservative child planes on a power-of-two grid
//   expand_planes     the quantized planes as floats rounded outward
//
// Every double product and sum is rounded on its own (BW_MUL / BW_ADD /
// BW_SUB: no fused multiply-add on the device), the divisions are IEEE and
// the rest (frexp, ldexp, floor, ceil, nextafterf) is exact, so host and
// device agree bit for bit.
#pragma once
#include <math.h>
#include <stdint.h>

#include "bvh_build.h"

#ifdef __CUDACC__
#define BW_HD __host__ __device__ inline
#else
#define BW_HD inline
#endif

// Double products and sums rounded one at a time on the device too (no
// fused multiply-add), as the host evaluates them.
#ifdef __CUDA_ARCH__
#define BW_MUL(a, b) __dmul_rn(a, b)
#define BW_ADD(a, b) __dadd_rn(a, b)
#define BW_SUB(a, b) __dsub_rn(a, b)
#else
#define BW_MUL(a, b) ((a) * (b))
#define BW_ADD(a, b) ((a) + (b))
#define BW_SUB(a, b) ((a) - (b))
#endif

namespace dort_gpu {

BW_HD double bw_area(const float lo[3], const float hi[3]) {
  if(!(lo[0] <= hi[0])) { return 0.0; }
  double x = BW_SUB(double(hi[0]), double(lo[0]));
  double y = BW_SUB(double(hi[1]), double(lo[1]));
  double z = BW_SUB(double(hi[2]), double(lo[2]));
  return BW_MUL(2.0, BW_ADD(BW_ADD(BW_MUL(x, y), BW_MUL(y, z)), BW_MUL(z, x)));
}

// Accessor A: bool leaf(b), uint32_t left(b), uint32_t right(b),
// const float* lo(b), const float* hi(b).  Returns the candidate count.
template<class A>
BW_HD uint32_t open_candidates(const A& acc, uint32_t node, uint32_t width, uint32_t cands[8]) {
  uint32_t n = 0;
  if(acc.leaf(node)) {
    cands[n++] = node;
  } else {
    cands[n++] = acc.left(node);
    cands[n++] = acc.right(node);
  }
  while(n < width) {
    int best = -1;
    double best_area = -1.0;
    for(uint32_t i = 0; i < n; ++i) {
      if(acc.leaf(cands[i])) { continue; }
      double a = bw_area(acc.lo(cands[i]), acc.hi(cands[i]));
      if(a > best_area) { best_area = a; best = int(i); }
    }
    if(best < 0) { break; }
    uint32_t b = cands[best];
    cands[best] = acc.left(b);
    cands[n++] = acc.right(b);
  }
  return n;
}

// Fills cand_in_slot[8] (candidate index or -1) and the node box.
template<class A>
BW_HD void assign_slots(const A& acc, const uint32_t* cands, uint32_t n, float nlo[3],
                        float nhi[3], int cand_in_slot[8]) {
  for(int a = 0; a < 3; ++a) { nlo[a] = INFINITY; nhi[a] = -INFINITY; }
  for(uint32_t c = 0; c < n; ++c) {
    const float* lo = acc.lo(cands[c]);
    const float* hi = acc.hi(cands[c]);
    for(int a = 0; a < 3; ++a) {
      nlo[a] = fminf(nlo[a], lo[a]);
      nhi[a] = fmaxf(nhi[a], hi[a]);
    }
  }
  double pc[3];
  for(int a = 0; a < 3; ++a) { pc[a] = BW_MUL(0.5, BW_ADD(double(nlo[a]), double(nhi[a]))); }
  bool slot_used[8] = {false, false, false, false, false, false, false, false};
  bool cand_done[8] = {false, false, false, false, false, false, false, false};
  for(int s = 0; s < 8; ++s) { cand_in_slot[s] = -1; }
  for(uint32_t k = 0; k < n; ++k) {
    double best = INFINITY;
    int bc = -1, bs = -1;
    for(uint32_t c = 0; c < n; ++c) {
      if(cand_done[c]) { continue; }
      const float* lo = acc.lo(cands[c]);
      const float* hi = acc.hi(cands[c]);
      double d[3];
      for(int a = 0; a < 3; ++a) {
        d[a] = BW_SUB(BW_MUL(0.5, BW_ADD(double(lo[a]), double(hi[a]))), pc[a]);
      }
      for(int s = 0; s < 8; ++s) {
        if(slot_used[s]) { continue; }
        double cost = BW_ADD(BW_ADD((s & 1) ? -d[0] : d[0], (s & 2) ? -d[1] : d[1]),
                             (s & 4) ? -d[2] : d[2]);
        if(cost < best) { best = cost; bc = int(c); bs = s; }
      }
    }
    cand_done[bc] = true;
    slot_used[bs] = true;
    cand_in_slot[bs] = bc;
  }
}

// Picks the quantization grid of one axis: step 2^e, origin p one step below
// the node's lower bound, 253 steps covering the extent; every child plane
// encloses its child with at least one step of margin.  Returns false if the
// exponent cannot be represented.
BW_HD bool quantize_axis(float node_lo, float node_hi, const float* clo, const float* chi,
                         int n, float& p_out, uint8_t& e_out, uint8_t* qlo, uint8_t* qhi) {
  double lo = node_lo, hi = node_hi;
  double ext = BW_SUB(hi, lo);
  double mag = fmax(fabs(lo), fabs(hi));
  double min_step = fmax(BW_MUL(mag, ldexp(1.0, -20)), ldexp(1.0, -100));
  double step = fmax(ext / 253.0, min_step);
  int ex;
  double m = frexp(step, &ex);       // step = m 2^ex, m in [0.5, 1)
  int e = m == 0.5 ? ex - 1 : ex;    // ceil(log2(step))
  for(int attempt = 0; attempt < 8; ++attempt, ++e) {
    if(e + 127 < 1 || e + 127 > 254) { return false; }
    double s = ldexp(1.0, e);
    double pd = BW_SUB(lo, s);
    float pf = float(pd);
    if(double(pf) > pd) { pf = nextafterf(pf, -INFINITY); }
    bool ok = true;
    for(int i = 0; i < n && ok; ++i) {
      double ql = BW_SUB(floor(BW_SUB(double(clo[i]), double(pf)) / s), 1.0);
      double qh = BW_ADD(ceil(BW_SUB(double(chi[i]), double(pf)) / s), 1.0);
      if(ql < 0.0 || qh > 255.0) { ok = false; break; }
      double margin = BW_MUL(s, 0.999);
      if(BW_ADD(double(pf), BW_MUL(ql, s)) > BW_SUB(double(clo[i]), margin) ||
         BW_ADD(double(pf), BW_MUL(qh, s)) < BW_ADD(double(chi[i]), margin)) {
        ok = false;
        break;
      }
      qlo[i] = uint8_t(ql);
      qhi[i] = uint8_t(qh);
    }
    if(ok) {
      p_out = pf;
      e_out = uint8_t(e + 127);
      return true;
    }
  }
  return false;
}

// Quantizes the 8 slot boxes of a node (empty slots: cand_in_slot < 0) into
// `node` (p, e, qlo, qhi); empty slots get an inverted box.
template<class A>
BW_HD bool quantize_node(const A& acc, const uint32_t* cands, const int cand_in_slot[8],
                         const float nlo[3], const float nhi[3], WideNode& node) {
  float clo[3][8], chi[3][8];
  for(int s = 0; s < 8; ++s) {
    int c = cand_in_slot[s];
    for(int a = 0; a < 3; ++a) {
      clo[a][s] = c >= 0 ? acc.lo(cands[c])[a] : nlo[a];
      chi[a][s] = c >= 0 ? acc.hi(cands[c])[a] : nlo[a];
    }
  }
  for(int a = 0; a < 3; ++a) {
    if(!quantize_axis(nlo[a], nhi[a], clo[a], chi[a], 8, node.p[a], node.e[a], node.qlo[a],
                      node.qhi[a])) {
      return false;
    }
  }
  for(int s = 0; s < 8; ++s) {
    if(cand_in_slot[s] < 0) {
      for(int a = 0; a < 3; ++a) { node.qlo[a][s] = 255; node.qhi[a][s] = 0; }
    }
  }
  return true;
}

// The float-plane form of a quantized node (planes rounded outward).
BW_HD void expand_planes(const WideNode& n, WideNodeF& f) {
  f.child_base = n.child_base;
  f.tri_base = n.tri_base;
  for(int k = 0; k < 8; ++k) { f.meta[k] = n.meta[k]; }
  f.imask = n.imask;
  f.pad[0] = f.pad[1] = f.pad[2] = 0;
  for(int a = 0; a < 3; ++a) {
    double s = ldexp(1.0, int(n.e[a]) - 127);
    for(int k = 0; k < 8; ++k) {
      double lo = BW_ADD(double(n.p[a]), BW_MUL(double(n.qlo[a][k]), s));
      double hi = BW_ADD(double(n.p[a]), BW_MUL(double(n.qhi[a][k]), s));
      float lf = float(lo), hf = float(hi);
      if(double(lf) > lo) { lf = nextafterf(lf, -INFINITY); }
      if(double(hf) < hi) { hf = nextafterf(hf, INFINITY); }
      f.pl[a][0][k] = lf;
      f.pl[a][1][k] = hf;
    }
  }
}

}  // namespace dort_gpu
