// Device construction of the wide BVH: a binary tree (binned SAH, top down;
// or Morton order + PLOC, bottom up), then a breadth-first collapse into wide
// nodes.  See bvh_device.h.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "bvh_device.h"
#include "bvh_wide.h"
#include "common.h"

namespace dort_gpu {
namespace {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr int kPlocRadius = 8;       // PLOC search radius (positions on each side)
constexpr int kNnBlock = 256;
constexpr uint32_t kMaxPlocIterations = 4096;
constexpr int kBins = 32;            // SAH bins per axis (as the host build)
constexpr uint32_t kChunk = 256;     // primitives binned by one warp
constexpr int kWarps = 4;            // warps per block of the SAH kernels
constexpr uint32_t kForceHalfDepth = 36;   // deeper binary nodes split by count
constexpr uint32_t kMaxSahLevels = 128;

// Binary node, 32 bytes: box, then the children (internal) or, for a leaf,
// kLeafBit | first position in the leaf-order array and the primitive count.
struct DevBin {
  float lo[3];
  float hi[3];
  uint32_t left, right;
};

struct DevAcc {
  const DevBin* n;
  __host__ __device__ bool leaf(uint32_t b) const { return (n[b].left & kLeafBit) != 0u; }
  __host__ __device__ uint32_t left(uint32_t b) const { return n[b].left; }
  __host__ __device__ uint32_t right(uint32_t b) const { return n[b].right; }
  __host__ __device__ const float* lo(uint32_t b) const { return n[b].lo; }
  __host__ __device__ const float* hi(uint32_t b) const { return n[b].hi; }
};

// Order-preserving float <-> uint encoding for atomicMin / atomicMax.
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float warp_min(float v) {
  for(int o = 16; o > 0; o >>= 1) { v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o)); }
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for(int o = 16; o > 0; o >>= 1) { v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o)); }
  return v;
}

// Triangle boxes and the bounds of all boxes (0..5) and centroids (6..11).
__global__ void k_prim_bounds(const float* __restrict__ verts, const uint32_t* __restrict__ tris,
                              uint32_t n, DevBin* __restrict__ prim,
                              uint32_t* __restrict__ bounds) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  float v[12];
  for(int a = 0; a < 3; ++a) {
    v[a] = v[6 + a] = INFINITY;
    v[3 + a] = v[9 + a] = -INFINITY;
  }
  if(t < n) {
    DevBin b;
    for(int a = 0; a < 3; ++a) { b.lo[a] = INFINITY; b.hi[a] = -INFINITY; }
    for(int k = 0; k < 3; ++k) {
      const float* p = verts + 3 * size_t(tris[3 * size_t(t) + k]);
      for(int a = 0; a < 3; ++a) {
        b.lo[a] = fminf(b.lo[a], p[a]);
        b.hi[a] = fmaxf(b.hi[a], p[a]);
      }
    }
    b.left = t | kLeafBit;
    b.right = 1;
    prim[t] = b;
    for(int a = 0; a < 3; ++a) {
      float c = __fmul_rn(0.5f, __fadd_rn(b.lo[a], b.hi[a]));
      v[a] = b.lo[a];
      v[3 + a] = b.hi[a];
      v[6 + a] = v[9 + a] = c;
    }
  }
  for(int a = 0; a < 3; ++a) {
    v[a] = warp_min(v[a]);
    v[3 + a] = warp_max(v[3 + a]);
    v[6 + a] = warp_min(v[6 + a]);
    v[9 + a] = warp_max(v[9 + a]);
  }
  if((threadIdx.x & 31) == 0 && v[0] <= v[3]) {
    for(int a = 0; a < 3; ++a) {
      atomicMin(&bounds[a], f2o(v[a]));
      atomicMax(&bounds[3 + a], f2o(v[3 + a]));
      atomicMin(&bounds[6 + a], f2o(v[6 + a]));
      atomicMax(&bounds[9 + a], f2o(v[9 + a]));
    }
  }
}

// ---- PLOC ----------------------------------------------------------------------

// Spreads the low 21 bits of x to every third bit.
__device__ __forceinline__ uint64_t spread21(uint32_t x) {
  uint64_t v = x & 0x1fffffu;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__global__ void k_morton(const DevBin* __restrict__ prim, uint32_t n,
                         const uint32_t* __restrict__ bounds, uint64_t* __restrict__ keys,
                         uint32_t* __restrict__ vals) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= n) { return; }
  uint64_t key = 0;
  for(int a = 0; a < 3; ++a) {
    float lo = o2f(bounds[6 + a]), hi = o2f(bounds[9 + a]);
    float ext = hi - lo;
    uint32_t q = 0;
    if(ext > 0.f) {
      float c = __fmul_rn(0.5f, __fadd_rn(prim[t].lo[a], prim[t].hi[a]));
      float f = (c - lo) / ext * 2097152.f;
      q = f >= 2097151.f ? 2097151u : (f > 0.f ? uint32_t(f) : 0u);
    }
    key |= spread21(q) << (2 - a);
  }
  keys[t] = key;
  vals[t] = t;
}

// Leaves in Morton order: node i holds leaf-order position i (triangle
// order[i]); cluster i = node i.
__global__ void k_leaves(const DevBin* __restrict__ prim, const uint32_t* __restrict__ order,
                         uint32_t n, DevBin* __restrict__ nodes, uint32_t* __restrict__ count,
                         uint32_t* __restrict__ clusters) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  DevBin b = prim[order[i]];
  b.left = i | kLeafBit;
  b.right = 1;
  nodes[i] = b;
  count[i] = 1;
  clusters[i] = i;
}

__device__ __forceinline__ float union_area(float alx, float aly, float alz, float ahx,
                                            float ahy, float ahz, float blx, float bly,
                                            float blz, float bhx, float bhy, float bhz) {
  float x = fmaxf(ahx, bhx) - fminf(alx, blx);
  float y = fmaxf(ahy, bhy) - fminf(aly, bly);
  float z = fmaxf(ahz, bhz) - fminf(alz, blz);
  return __fmul_rn(2.f, __fadd_rn(__fadd_rn(__fmul_rn(x, y), __fmul_rn(y, z)), __fmul_rn(z, x)));
}

// Symmetric 32-bit mix of a pair of positions: orders pairs of equal union
// area pseudo-randomly, so that inputs with many identical boxes still form
// many mutual pairs per iteration (ties broken by position alone would pair
// only the first two of a run of equal boxes).
__device__ __forceinline__ uint32_t pair_hash(uint32_t a, uint32_t b) {
  uint32_t lo = min(a, b), hi = max(a, b);
  uint32_t h = lo * 0x9e3779b1u ^ (hi + 0x7f4a7c15u) * 0x85ebca77u;
  h ^= h >> 15;
  h *= 0x2c1b3c6du;
  h ^= h >> 12;
  h *= 0x297a2d39u;
  h ^= h >> 15;
  return h;
}

// Nearest neighbour of every cluster within kPlocRadius positions: the one
// whose union box has the smallest area, then the smallest pair_hash, then
// the smallest position.  Every part of that order is symmetric in the pair,
// so the pair that is first in it overall is always mutual: each iteration
// merges at least one pair.
__global__ void __launch_bounds__(kNnBlock) k_nearest(const DevBin* __restrict__ nodes,
                                                      const uint32_t* __restrict__ clusters,
                                                      uint32_t m, uint32_t* __restrict__ nn) {
  __shared__ float s[6][kNnBlock + 2 * kPlocRadius];
  int base = int(blockIdx.x) * kNnBlock - kPlocRadius;
  for(int k = threadIdx.x; k < kNnBlock + 2 * kPlocRadius; k += blockDim.x) {
    int i = base + k;
    if(i >= 0 && uint32_t(i) < m) {
      const DevBin& b = nodes[clusters[i]];
      s[0][k] = b.lo[0]; s[1][k] = b.lo[1]; s[2][k] = b.lo[2];
      s[3][k] = b.hi[0]; s[4][k] = b.hi[1]; s[5][k] = b.hi[2];
    }
  }
  __syncthreads();
  uint32_t i = blockIdx.x * kNnBlock + threadIdx.x;
  if(i >= m) { return; }
  int li = int(threadIdx.x) + kPlocRadius;
  float alx = s[0][li], aly = s[1][li], alz = s[2][li];
  float ahx = s[3][li], ahy = s[4][li], ahz = s[5][li];
  uint64_t best = ~0ull;
  uint32_t best_j = ~0u;
  for(int d = -kPlocRadius; d <= kPlocRadius; ++d) {
    if(d == 0) { continue; }
    int j = int(i) + d;
    if(j < 0 || uint32_t(j) >= m) { continue; }
    int lj = li + d;
    float a = union_area(alx, aly, alz, ahx, ahy, ahz, s[0][lj], s[1][lj], s[2][lj], s[3][lj],
                         s[4][lj], s[5][lj]);
    uint64_t key = (uint64_t(__float_as_uint(a)) << 32) | pair_hash(i, uint32_t(j));
    if(key < best || (key == best && uint32_t(j) < best_j)) {
      best = key;
      best_j = uint32_t(j);
    }
  }
  nn[i] = best_j;
}

// Per position: low word 1 if the position survives (unmerged, or the lower
// position of a merged pair), high word 1 if it becomes a new node.
__global__ void k_merge_flags(const uint32_t* __restrict__ nn, uint32_t m,
                              uint64_t* __restrict__ flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= m) { return; }
  uint32_t j = nn[i];
  bool mutual = nn[j] == i;
  uint64_t f;
  if(!mutual) { f = 1; }
  else if(i < j) { f = 1 | (1ull << 32); }
  else { f = 0; }
  flags[i] = f;
}

__global__ void k_merge(DevBin* __restrict__ nodes, uint32_t* __restrict__ count,
                        const uint32_t* __restrict__ clusters, const uint32_t* __restrict__ nn,
                        const uint64_t* __restrict__ flags, const uint64_t* __restrict__ incl,
                        uint32_t m, uint32_t next, uint32_t* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= m) { return; }
  uint64_t f = flags[i];
  if(f == 0) { return; }
  uint64_t ex = incl[i] - f;
  uint32_t pos = uint32_t(ex);
  if(f >> 32) {
    uint32_t nid = next + uint32_t(ex >> 32);
    uint32_t a = clusters[i], b = clusters[nn[i]];
    DevBin na = nodes[a], nb = nodes[b];
    DevBin r;
    for(int k = 0; k < 3; ++k) {
      r.lo[k] = fminf(na.lo[k], nb.lo[k]);
      r.hi[k] = fmaxf(na.hi[k], nb.hi[k]);
    }
    r.left = a;
    r.right = b;
    nodes[nid] = r;
    count[nid] = count[a] + count[b];
    out[pos] = nid;
  } else {
    out[pos] = clusters[i];
  }
}

// ---- binned SAH, top down, one level of the binary tree per round ------------------
//
// Every open node ("task") owns the range [begin, begin + count) of the
// primitive index array.  A round bins every task's primitives (one warp per
// chunk of kChunk primitives; a task of several chunks merges its warps' bins
// in global memory and its last warp evaluates them), picks each task's split
// (or makes it a leaf) as the host builder does (32 bins on each axis, cost
// 1 + (A_l n_l + A_r n_r) / A against n), partitions the ranges stably by a
// prefix sum of the left-side flags, and opens the children as the next
// round's tasks.

struct Task {
  uint32_t node, begin, count, depth;
  float lo[3], hi[3];     // box of the primitives
  float clo[3], chi[3];   // bounds of their centroids
};

struct Split {
  int32_t axis;           // -1: split the range in two halves by count
  int32_t bin;            // left = bins 0..bin on `axis`
  uint32_t lcount;
  uint32_t leaf;
};

constexpr int kBinWords = 3 * kBins * 7;   // count, lo[3], hi[3] per bin and axis

__device__ __forceinline__ int bin_of(float c, float clo, float k) {
  int b = int(__fmul_rn(__fsub_rn(c, clo), k));
  return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}

__device__ __forceinline__ float bin_scale(float clo, float chi) {
  float ext = chi - clo;
  return ext > 0.f ? float(kBins) / ext : 0.f;
}

__device__ __forceinline__ double box_area_d(float lx, float ly, float lz, float hx, float hy,
                                             float hz) {
  if(!(lx <= hx)) { return 0.0; }
  double x = double(hx) - lx, y = double(hy) - ly, z = double(hz) - lz;
  return 2.0 * (x * y + y * z + z * x);
}

__device__ __forceinline__ uint32_t bin_init(int w) {
  int f = w % 7;
  return f == 0 ? 0u : (f <= 3 ? 0xffffffffu : 0u);
}

__global__ void k_task_chunks(const Task* __restrict__ tasks, uint32_t T,
                              uint64_t* __restrict__ packed) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= T) { return; }
  uint32_t chunks = (tasks[t].count + kChunk - 1) / kChunk;
  packed[t] = uint64_t(chunks) | (uint64_t(chunks > 1 ? 1u : 0u) << 32);
}

__global__ void k_expand(const Task* __restrict__ tasks, uint32_t T,
                         const uint64_t* __restrict__ packed, const uint64_t* __restrict__ incl,
                         uint32_t* __restrict__ chunk_task, uint32_t* __restrict__ chunk_part,
                         uint32_t* __restrict__ bin_slot, uint32_t* __restrict__ gbins,
                         uint32_t* __restrict__ gcounter, uint32_t* __restrict__ acc) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= T) { return; }
  uint64_t ex = incl[t] - packed[t];
  uint32_t first = uint32_t(ex), chunks = uint32_t(packed[t]);
  for(uint32_t j = 0; j < chunks; ++j) {
    chunk_task[first + j] = t;
    chunk_part[first + j] = j;
  }
  uint32_t slot = ~0u;
  if(chunks > 1) {
    slot = uint32_t(ex >> 32);
    uint32_t* g = gbins + size_t(slot) * kBinWords;
    for(int w = 0; w < kBinWords; ++w) { g[w] = bin_init(w); }
    gcounter[slot] = 0;
  }
  bin_slot[t] = slot;
  // child box / centroid-bound accumulators: [side][lo3 hi3 clo3 chi3]
  for(int s = 0; s < 2; ++s) {
    for(int w = 0; w < 12; ++w) {
      acc[24 * size_t(t) + 12 * s + w] = ((w / 3) % 2 == 0) ? 0xffffffffu : 0u;
    }
  }
}

// The split of one task from its bins (shared memory of one warp); lane 0
// writes it.
__device__ void evaluate_split(const uint32_t* __restrict__ bins, const Task& task,
                               uint32_t max_leaf, Split* __restrict__ out) {
  int lane = threadIdx.x & 31;
  double best = INFINITY;
  int best_axis = -1, best_bin = 0;
  uint32_t best_l = 0;
  bool force_half = task.depth >= kForceHalfDepth;
  for(int a = 0; a < 3 && !force_half; ++a) {
    if(!(task.chi[a] - task.clo[a] > 0.f)) { continue; }
    const uint32_t* b = bins + (a * kBins + lane) * 7;
    uint32_t cnt = b[0];
    float lo[3], hi[3];
    for(int k = 0; k < 3; ++k) {
      lo[k] = cnt ? o2f(b[1 + k]) : INFINITY;
      hi[k] = cnt ? o2f(b[4 + k]) : -INFINITY;
    }
    // inclusive prefix (bins 0..lane) and suffix (bins lane..31)
    uint32_t pc = cnt, sc = cnt;
    float pl[3] = {lo[0], lo[1], lo[2]}, ph[3] = {hi[0], hi[1], hi[2]};
    float sl[3] = {lo[0], lo[1], lo[2]}, sh[3] = {hi[0], hi[1], hi[2]};
    for(int o = 1; o < 32; o <<= 1) {
      uint32_t upc = __shfl_up_sync(0xffffffffu, pc, o);
      uint32_t dsc = __shfl_down_sync(0xffffffffu, sc, o);
      float u[6], d[6];
      for(int k = 0; k < 3; ++k) {
        u[k] = __shfl_up_sync(0xffffffffu, pl[k], o);
        u[3 + k] = __shfl_up_sync(0xffffffffu, ph[k], o);
        d[k] = __shfl_down_sync(0xffffffffu, sl[k], o);
        d[3 + k] = __shfl_down_sync(0xffffffffu, sh[k], o);
      }
      if(lane >= o) {
        pc += upc;
        for(int k = 0; k < 3; ++k) { pl[k] = fminf(pl[k], u[k]); ph[k] = fmaxf(ph[k], u[3 + k]); }
      }
      if(lane + o < 32) {
        sc += dsc;
        for(int k = 0; k < 3; ++k) { sl[k] = fminf(sl[k], d[k]); sh[k] = fmaxf(sh[k], d[3 + k]); }
      }
    }
    // split after bin `lane`: left = prefix(lane), right = suffix(lane + 1)
    uint32_t rc = __shfl_down_sync(0xffffffffu, sc, 1);
    float rl[3], rh[3];
    for(int k = 0; k < 3; ++k) {
      rl[k] = __shfl_down_sync(0xffffffffu, sl[k], 1);
      rh[k] = __shfl_down_sync(0xffffffffu, sh[k], 1);
    }
    double cost = INFINITY;
    if(lane < 31 && pc > 0 && rc > 0) {
      cost = box_area_d(pl[0], pl[1], pl[2], ph[0], ph[1], ph[2]) * pc +
             box_area_d(rl[0], rl[1], rl[2], rh[0], rh[1], rh[2]) * rc;
    }
    // the first minimum in bin order on this axis, then across axes in order
    double c = cost;
    int bi = lane;
    for(int o = 16; o > 0; o >>= 1) {
      double oc = __shfl_xor_sync(0xffffffffu, c, o);
      int ob = __shfl_xor_sync(0xffffffffu, bi, o);
      if(oc < c || (oc == c && ob < bi)) { c = oc; bi = ob; }
    }
    uint32_t lc = __shfl_sync(0xffffffffu, pc, bi);
    if(c < best) { best = c; best_axis = a; best_bin = bi; best_l = lc; }
  }
  if(lane != 0) { return; }
  Split s;
  s.axis = best_axis;
  s.bin = best_bin;
  s.lcount = best_l;
  s.leaf = 0;
  double parent = fmax(box_area_d(task.lo[0], task.lo[1], task.lo[2], task.hi[0], task.hi[1],
                                  task.hi[2]), 1e-300);
  double split_cost = kSahTraversal + best / parent;
  double leaf_cost = double(task.count);
  if(task.count <= max_leaf && (best_axis < 0 || leaf_cost <= split_cost)) {
    s.leaf = 1;
  } else if(best_axis < 0) {
    s.axis = -1;
    s.lcount = task.count / 2;
  }
  *out = s;
}

__global__ void __launch_bounds__(32 * kWarps)
k_bin_split(const DevBin* __restrict__ prim, const uint32_t* __restrict__ idx,
            const Task* __restrict__ tasks, const uint32_t* __restrict__ chunk_task,
            const uint32_t* __restrict__ chunk_part, uint32_t C,
            const uint32_t* __restrict__ bin_slot, uint32_t* __restrict__ gbins,
            uint32_t* __restrict__ gcounter, uint32_t max_leaf, Split* __restrict__ splits) {
  __shared__ uint32_t sbins[kWarps][kBinWords];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t c = blockIdx.x * kWarps + w;
  if(c >= C) { return; }
  uint32_t* bins = sbins[w];
  for(int k = lane; k < kBinWords; k += 32) { bins[k] = bin_init(k); }
  __syncwarp();
  uint32_t t = chunk_task[c];
  const Task task = tasks[t];
  uint32_t begin = task.begin + chunk_part[c] * kChunk;
  uint32_t end = min(begin + kChunk, task.begin + task.count);
  float k3[3];
  for(int a = 0; a < 3; ++a) { k3[a] = bin_scale(task.clo[a], task.chi[a]); }
  for(uint32_t i = begin + lane; i < end; i += 32) {
    const DevBin b = prim[idx[i]];
    for(int a = 0; a < 3; ++a) {
      if(k3[a] == 0.f) { continue; }
      float cc = __fmul_rn(0.5f, __fadd_rn(b.lo[a], b.hi[a]));
      uint32_t* e = bins + (a * kBins + bin_of(cc, task.clo[a], k3[a])) * 7;
      atomicAdd(&e[0], 1u);
      for(int q = 0; q < 3; ++q) {
        atomicMin(&e[1 + q], f2o(b.lo[q]));
        atomicMax(&e[4 + q], f2o(b.hi[q]));
      }
    }
  }
  __syncwarp();
  uint32_t chunks = (task.count + kChunk - 1) / kChunk;
  if(chunks == 1) {
    evaluate_split(bins, task, max_leaf, &splits[t]);
    return;
  }
  uint32_t slot = bin_slot[t];
  uint32_t* g = gbins + size_t(slot) * kBinWords;
  for(int k = lane; k < kBinWords; k += 32) {
    int f = k % 7;
    uint32_t v = bins[k];
    if(f == 0) { if(v) { atomicAdd(&g[k], v); } }
    else if(f <= 3) { if(v != 0xffffffffu) { atomicMin(&g[k], v); } }
    else if(v) { atomicMax(&g[k], v); }
  }
  __threadfence();
  __syncwarp();
  uint32_t done = 0;
  if(lane == 0) { done = atomicAdd(&gcounter[slot], 1u); }
  done = __shfl_sync(0xffffffffu, done, 0);
  if(done != chunks - 1) { return; }
  // the last warp of the task: every other warp's bins are in g
  __threadfence();
  for(int k = lane; k < kBinWords; k += 32) { bins[k] = __ldcg(&g[k]); }
  __syncwarp();
  evaluate_split(bins, task, max_leaf, &splits[t]);
}

__device__ __forceinline__ bool goes_left(const DevBin& b, const Task& task, const Split& s,
                                          uint32_t pos) {
  if(s.axis < 0) { return pos - task.begin < s.lcount; }
  int a = s.axis;
  float cc = __fmul_rn(0.5f, __fadd_rn(b.lo[a], b.hi[a]));
  return bin_of(cc, task.clo[a], bin_scale(task.clo[a], task.chi[a])) <= s.bin;
}

__global__ void __launch_bounds__(32 * kWarps)
k_partition(const DevBin* __restrict__ prim, const uint32_t* __restrict__ idx,
            const Task* __restrict__ tasks, const uint32_t* __restrict__ chunk_task,
            const uint32_t* __restrict__ chunk_part, uint32_t C,
            const Split* __restrict__ splits, uint32_t* __restrict__ flags) {
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t c = blockIdx.x * kWarps + w;
  if(c >= C) { return; }
  uint32_t t = chunk_task[c];
  const Task task = tasks[t];
  const Split s = splits[t];
  uint32_t begin = task.begin + chunk_part[c] * kChunk;
  uint32_t end = min(begin + kChunk, task.begin + task.count);
  for(uint32_t i = begin + lane; i < end; i += 32) {
    flags[i] = (!s.leaf && goes_left(prim[idx[i]], task, s, i)) ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(32 * kWarps)
k_scatter(const DevBin* __restrict__ prim, const uint32_t* __restrict__ idx,
          uint32_t* __restrict__ idx2, uint32_t* __restrict__ final_idx,
          const Task* __restrict__ tasks, const uint32_t* __restrict__ chunk_task,
          const uint32_t* __restrict__ chunk_part, uint32_t C, const Split* __restrict__ splits,
          const uint32_t* __restrict__ flags, const uint32_t* __restrict__ scan,
          uint32_t* __restrict__ acc) {
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t c = blockIdx.x * kWarps + w;
  if(c >= C) { return; }
  uint32_t t = chunk_task[c];
  const Task task = tasks[t];
  const Split s = splits[t];
  uint32_t begin = task.begin + chunk_part[c] * kChunk;
  uint32_t end = min(begin + kChunk, task.begin + task.count);
  if(s.leaf) {
    for(uint32_t i = begin + lane; i < end; i += 32) { final_idx[i] = idx[i]; }
    return;
  }
  uint32_t base = scan[task.begin];
  uint32_t rcount = task.count - s.lcount;
  float v[2][12];
  for(int side = 0; side < 2; ++side) {
    for(int q = 0; q < 12; ++q) { v[side][q] = ((q / 3) % 2 == 0) ? INFINITY : -INFINITY; }
  }
  for(uint32_t i = begin + lane; i < end; i += 32) {
    uint32_t p = idx[i];
    const DevBin b = prim[p];
    bool left = flags[i] != 0u;
    uint32_t lrank = scan[i] - base;
    uint32_t pos = left ? task.begin + lrank : task.begin + s.lcount + (i - task.begin - lrank);
    if(pos >= task.begin + task.count) { continue; }   // cannot happen: counts agree
    idx2[pos] = p;
    if((left && s.lcount == 1) || (!left && rcount == 1)) { final_idx[pos] = p; }
    int side = left ? 0 : 1;
    for(int a = 0; a < 3; ++a) {
      float cc = __fmul_rn(0.5f, __fadd_rn(b.lo[a], b.hi[a]));
      v[side][a] = fminf(v[side][a], b.lo[a]);
      v[side][3 + a] = fmaxf(v[side][3 + a], b.hi[a]);
      v[side][6 + a] = fminf(v[side][6 + a], cc);
      v[side][9 + a] = fmaxf(v[side][9 + a], cc);
    }
  }
  for(int side = 0; side < 2; ++side) {
    for(int q = 0; q < 12; ++q) {
      bool is_min = (q / 3) % 2 == 0;
      float r = is_min ? warp_min(v[side][q]) : warp_max(v[side][q]);
      if(lane == 0 && r != (is_min ? INFINITY : -INFINITY)) {
        uint32_t* dst = &acc[24 * size_t(t) + 12 * side + q];
        if(is_min) { atomicMin(dst, f2o(r)); } else { atomicMax(dst, f2o(r)); }
      }
    }
  }
}

// Per task: low word = binary nodes to allocate (2 for a split), high word =
// tasks to open (the children with more than one primitive).
__global__ void k_child_counts(const Task* __restrict__ tasks, uint32_t T,
                               const Split* __restrict__ splits, uint64_t* __restrict__ packed) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= T) { return; }
  const Split s = splits[t];
  uint64_t v = 0;
  if(!s.leaf) {
    uint32_t open = (s.lcount > 1 ? 1u : 0u) + (tasks[t].count - s.lcount > 1 ? 1u : 0u);
    v = 2u | (uint64_t(open) << 32);
  }
  packed[t] = v;
}

__global__ void k_children(const Task* __restrict__ tasks, uint32_t T,
                           const Split* __restrict__ splits, const uint64_t* __restrict__ packed,
                           const uint64_t* __restrict__ incl, const uint32_t* __restrict__ acc,
                           uint32_t node_base, DevBin* __restrict__ nodes,
                           uint32_t* __restrict__ count, Task* __restrict__ next) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= T) { return; }
  const Task task = tasks[t];
  const Split s = splits[t];
  DevBin me;
  for(int a = 0; a < 3; ++a) { me.lo[a] = task.lo[a]; me.hi[a] = task.hi[a]; }
  count[task.node] = task.count;
  if(s.leaf) {
    me.left = kLeafBit | task.begin;
    me.right = task.count;
    nodes[task.node] = me;
    return;
  }
  uint64_t ex = incl[t] - packed[t];
  uint32_t c0 = node_base + uint32_t(ex);
  uint32_t slot = uint32_t(ex >> 32);
  me.left = c0;
  me.right = c0 + 1;
  nodes[task.node] = me;
  for(int side = 0; side < 2; ++side) {
    const uint32_t* v = acc + 24 * size_t(t) + 12 * side;
    uint32_t cnt = side == 0 ? s.lcount : task.count - s.lcount;
    uint32_t beg = side == 0 ? task.begin : task.begin + s.lcount;
    uint32_t id = c0 + side;
    if(cnt == 1) {
      DevBin b;
      for(int a = 0; a < 3; ++a) { b.lo[a] = o2f(v[a]); b.hi[a] = o2f(v[3 + a]); }
      b.left = kLeafBit | beg;
      b.right = 1;
      nodes[id] = b;
      count[id] = 1;
      continue;
    }
    Task ch;
    ch.node = id;
    ch.begin = beg;
    ch.count = cnt;
    ch.depth = task.depth + 1;
    for(int a = 0; a < 3; ++a) {
      ch.lo[a] = o2f(v[a]);
      ch.hi[a] = o2f(v[3 + a]);
      ch.clo[a] = o2f(v[6 + a]);
      ch.chi[a] = o2f(v[9 + a]);
    }
    next[slot++] = ch;
  }
}

__global__ void k_iota(uint32_t* __restrict__ a, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { a[i] = i; }
}

// ---- collapse ---------------------------------------------------------------------

struct Plan {
  uint32_t slot_node[8];   // binary node per slot, or ~0u
};

__device__ __forceinline__ bool slot_is_leaf(const DevAcc& acc, const uint32_t* count,
                                             uint32_t b, uint32_t max_leaf) {
  return acc.leaf(b) || count[b] <= max_leaf;
}

__global__ void k_plan(const DevBin* __restrict__ nodes, const uint32_t* __restrict__ count,
                       const uint32_t* __restrict__ qbin, uint32_t items, uint32_t width,
                       uint32_t max_leaf, Plan* __restrict__ plans,
                       uint64_t* __restrict__ counts) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= items) { return; }
  DevAcc acc{nodes};
  uint32_t cands[8];
  uint32_t n = open_candidates(acc, qbin[i], width, cands);
  float nlo[3], nhi[3];
  int cis[8];
  assign_slots(acc, cands, n, nlo, nhi, cis);
  Plan p;
  uint32_t ci = 0, lt = 0;
  for(int s = 0; s < 8; ++s) {
    uint32_t b = cis[s] >= 0 ? cands[cis[s]] : ~0u;
    p.slot_node[s] = b;
    if(b == ~0u) { continue; }
    if(slot_is_leaf(acc, count, b, max_leaf)) { lt += count[b]; } else { ci += 1; }
  }
  plans[i] = p;
  counts[i] = uint64_t(ci) | (uint64_t(lt) << 32);
}

template<bool kFloatPlanes>
__global__ void k_emit(const DevBin* __restrict__ nodes, const uint32_t* __restrict__ count,
                       const uint32_t* __restrict__ leaf_idx,
                       const float* __restrict__ verts, const uint32_t* __restrict__ tris,
                       const uint32_t* __restrict__ qbin, const uint32_t* __restrict__ qwide,
                       uint32_t items, uint32_t max_leaf, const Plan* __restrict__ plans,
                       const uint64_t* __restrict__ counts, const uint64_t* __restrict__ incl,
                       uint32_t wide_base, uint32_t tri_base0, void* __restrict__ wide_out,
                       LeafTri* __restrict__ leaf_out, uint32_t* __restrict__ qbin_next,
                       uint32_t* __restrict__ qwide_next, uint32_t* __restrict__ error) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= items) { return; }
  DevAcc acc{nodes};
  Plan p = plans[i];
  uint64_t ex = incl[i] - counts[i];
  uint32_t child_base = wide_base + uint32_t(ex);
  uint32_t next_pos = uint32_t(ex);
  uint32_t tri_base = tri_base0 + uint32_t(ex >> 32);
  uint32_t tri_room = uint32_t(counts[i] >> 32);   // leaf triangles this node owns

  uint32_t cands[8];
  int cis[8];
  float nlo[3] = {INFINITY, INFINITY, INFINITY}, nhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for(int s = 0; s < 8; ++s) {
    cands[s] = p.slot_node[s];
    cis[s] = p.slot_node[s] != ~0u ? s : -1;
    if(cis[s] >= 0) {
      for(int a = 0; a < 3; ++a) {
        nlo[a] = fminf(nlo[a], nodes[cands[s]].lo[a]);
        nhi[a] = fmaxf(nhi[a], nodes[cands[s]].hi[a]);
      }
    }
  }
  WideNode node;
  memset(&node, 0, sizeof(node));
  if(!quantize_node(acc, cands, cis, nlo, nhi, node)) {
    atomicOr(error, 1u);
    return;
  }
  node.child_base = child_base;
  node.tri_base = tri_base;
  uint32_t tri_off = 0, k_internal = 0;
  for(int s = 0; s < 8; ++s) {
    uint32_t b = p.slot_node[s];
    if(b == ~0u) { node.meta[s] = 0; continue; }
    if(!slot_is_leaf(acc, count, b, max_leaf)) {
      node.imask |= uint8_t(1u << s);
      node.meta[s] = uint8_t(0x20 | (24 + s));
      qbin_next[next_pos + k_internal] = b;
      qwide_next[next_pos + k_internal] = child_base + k_internal;
      ++k_internal;
      continue;
    }
    // leaf slot: the subtree's triangles, left first (at most max_leaf <= 3)
    uint32_t stack[8];
    int sp = 0;
    stack[sp++] = b;
    uint32_t cnt = 0;
    while(sp > 0) {
      uint32_t x = stack[--sp];
      if(acc.leaf(x)) {
        uint32_t first = nodes[x].left & ~kLeafBit, m = nodes[x].right;
        for(uint32_t k = 0; k < m && k < 4; ++k) {
          uint32_t t = leaf_idx[first + k];
          LeafTri lt;
          const float* p0 = verts + 3 * size_t(tris[3 * size_t(t)]);
          const float* p1 = verts + 3 * size_t(tris[3 * size_t(t) + 1]);
          const float* p2 = verts + 3 * size_t(tris[3 * size_t(t) + 2]);
          for(int a = 0; a < 3; ++a) {
            lt.p0[a] = p0[a];
            lt.e1[a] = __fsub_rn(p1[a], p0[a]);
            lt.e2[a] = __fsub_rn(p2[a], p0[a]);
          }
          lt.id = t;
          lt.pad1 = 0.f;
          lt.pad2 = 0.f;
          if(tri_off + cnt < tri_room) { leaf_out[tri_base + tri_off + cnt] = lt; }
          ++cnt;
        }
        if(m > 3) { cnt = 4; }   // rejected below
      } else if(sp + 2 <= 8) {
        stack[sp++] = nodes[x].right;
        stack[sp++] = nodes[x].left;
      } else {
        atomicOr(error, 2u);
        return;
      }
    }
    if(cnt == 0 || cnt > 3 || tri_off + cnt > 24 || tri_off + cnt > tri_room) {
      atomicOr(error, 2u);
      return;
    }
    node.meta[s] = uint8_t((((1u << cnt) - 1u) << 5) | tri_off);
    tri_off += cnt;
  }
  uint32_t w = qwide[i];
  if(kFloatPlanes) {
    WideNodeF f;
    expand_planes(node, f);
    static_cast<WideNodeF*>(wide_out)[w] = f;
  } else {
    static_cast<WideNode*>(wide_out)[w] = node;
  }
}

// Device buffers of one build, freed together.
struct Scratch {
  std::vector<void*> bufs;
  template<class T>
  T* alloc(size_t count, std::string& err) {
    void* p = nullptr;
    if(dev_alloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      err = "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed (BVH build)";
      return nullptr;
    }
    bufs.push_back(p);
    return static_cast<T*>(p);
  }
  ~Scratch() {
    for(void* p : bufs) { cudaFree(p); }
  }
};

inline uint32_t blocks_for(uint64_t n, uint32_t bs) { return uint32_t((n + bs - 1) / bs); }

bool cuda_ok(cudaError_t e, const char* what, std::string& err) {
  if(e == cudaSuccess) { return true; }
  err = std::string(what) + " failed: " + cudaGetErrorString(e);
  return false;
}

struct PinnedWords {
  uint64_t* p = nullptr;
  ~PinnedWords() { if(p) { cudaFreeHost(p); } }
};

// Inclusive sum of `count` packed words; the total lands in *host_total.
bool scan_total(void* temp, size_t temp_bytes, const uint64_t* in, uint64_t* out,
                uint32_t count, cudaStream_t st, uint64_t* host_total, std::string& err) {
  return cuda_ok(cub::DeviceScan::InclusiveSum(temp, temp_bytes, in, out, int(count), st),
                 "prefix sum", err) &&
         cuda_ok(cudaMemcpyAsync(host_total, out + (count - 1), sizeof(uint64_t),
                                 cudaMemcpyDeviceToHost, st), "counter read", err) &&
         cuda_ok(cudaStreamSynchronize(st), "BVH build", err);
}

// The binary tree: nodes, per-node triangle counts, leaf order, root.
struct BinTree {
  DevBin* nodes = nullptr;
  uint32_t* count = nullptr;
  uint32_t* leaf_idx = nullptr;
  uint32_t node_count = 0;
  uint32_t root = 0;
  uint32_t iterations = 0;
};

float decode_ordered(uint32_t u) {
  uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

bool build_ploc(Scratch& sc, const DevBin* prim, const uint32_t* bounds, uint32_t n,
                cudaStream_t st, void* temp, size_t temp_bytes, uint64_t* h_total,
                BinTree& bt, std::string& err) {
  uint32_t total_nodes = 2 * n - 1;
  uint64_t* keys = sc.alloc<uint64_t>(n, err);
  uint64_t* keys2 = sc.alloc<uint64_t>(n, err);
  uint32_t* vals = sc.alloc<uint32_t>(n, err);
  uint32_t* order = sc.alloc<uint32_t>(n, err);
  DevBin* nodes = sc.alloc<DevBin>(total_nodes, err);
  uint32_t* count = sc.alloc<uint32_t>(total_nodes, err);
  uint32_t* cl = sc.alloc<uint32_t>(n, err);
  uint32_t* cl2 = sc.alloc<uint32_t>(n, err);
  uint32_t* nn = sc.alloc<uint32_t>(n, err);
  uint64_t* flags = sc.alloc<uint64_t>(n, err);
  uint64_t* incl = sc.alloc<uint64_t>(n, err);
  if(!keys || !keys2 || !vals || !order || !nodes || !count || !cl || !cl2 || !nn || !flags ||
     !incl) {
    return false;
  }
  k_morton<<<blocks_for(n, 256), 256, 0, st>>>(prim, n, bounds, keys, vals);
  size_t tb = temp_bytes;
  if(!cuda_ok(cub::DeviceRadixSort::SortPairs(temp, tb, keys, keys2, vals, order, int(n), 0, 63,
                                              st), "radix sort", err)) {
    return false;
  }
  k_leaves<<<blocks_for(n, 256), 256, 0, st>>>(prim, order, n, nodes, count, cl);
  uint32_t m = n, next = n, iters = 0;
  while(m > 1) {
    if(++iters > kMaxPlocIterations) {
      err = "internal error: PLOC did not converge";
      return false;
    }
    k_nearest<<<blocks_for(m, kNnBlock), kNnBlock, 0, st>>>(nodes, cl, m, nn);
    k_merge_flags<<<blocks_for(m, 256), 256, 0, st>>>(nn, m, flags);
    tb = temp_bytes;
    if(!cuda_ok(cub::DeviceScan::InclusiveSum(temp, tb, flags, incl, int(m), st), "prefix sum",
                err)) {
      return false;
    }
    k_merge<<<blocks_for(m, 256), 256, 0, st>>>(nodes, count, cl, nn, flags, incl, m, next, cl2);
    if(!cuda_ok(cudaMemcpyAsync(h_total, incl + (m - 1), sizeof(uint64_t),
                                cudaMemcpyDeviceToHost, st), "counter read", err) ||
       !cuda_ok(cudaStreamSynchronize(st), "PLOC iteration", err)) {
      return false;
    }
    uint32_t m2 = uint32_t(*h_total);
    uint32_t made = uint32_t(*h_total >> 32);
    if(m2 >= m || made == 0 || next + made > total_nodes) {
      err = "internal error: PLOC made no progress";
      return false;
    }
    next += made;
    m = m2;
    std::swap(cl, cl2);
  }
  bt.nodes = nodes;
  bt.count = count;
  bt.leaf_idx = order;
  bt.node_count = next;
  bt.root = n == 1 ? 0u : next - 1;
  bt.iterations = iters;
  return true;
}

bool build_sah(Scratch& sc, const DevBin* prim, const uint32_t* d_bounds, uint32_t n,
               uint32_t max_leaf, cudaStream_t st, void* temp, size_t temp_bytes,
               uint64_t* h_total, BinTree& bt, std::string& err) {
  uint32_t total_nodes = 2 * n - 1;
  uint32_t task_cap = n / 2 + 2;                   // open tasks hold >= 2 primitives each
  uint32_t chunk_cap = task_cap + n / kChunk + 2;
  uint32_t slot_cap = n / (kChunk + 1) + 2;        // tasks of more than one chunk
  DevBin* nodes = sc.alloc<DevBin>(total_nodes, err);
  uint32_t* count = sc.alloc<uint32_t>(total_nodes, err);
  uint32_t* idx = sc.alloc<uint32_t>(n, err);
  uint32_t* idx2 = sc.alloc<uint32_t>(n, err);
  uint32_t* final_idx = sc.alloc<uint32_t>(n, err);
  uint32_t* flags = sc.alloc<uint32_t>(n, err);
  uint32_t* scan = sc.alloc<uint32_t>(n, err);
  Task* tasks = sc.alloc<Task>(task_cap, err);
  Task* tasks2 = sc.alloc<Task>(task_cap, err);
  Split* splits = sc.alloc<Split>(task_cap, err);
  uint64_t* packed = sc.alloc<uint64_t>(task_cap, err);
  uint64_t* incl = sc.alloc<uint64_t>(task_cap, err);
  uint32_t* acc = sc.alloc<uint32_t>(24 * size_t(task_cap), err);
  uint32_t* chunk_task = sc.alloc<uint32_t>(chunk_cap, err);
  uint32_t* chunk_part = sc.alloc<uint32_t>(chunk_cap, err);
  uint32_t* bin_slot = sc.alloc<uint32_t>(task_cap, err);
  uint32_t* gbins = sc.alloc<uint32_t>(size_t(slot_cap) * kBinWords, err);
  uint32_t* gcounter = sc.alloc<uint32_t>(slot_cap, err);
  if(!nodes || !count || !idx || !idx2 || !final_idx || !flags || !scan || !tasks || !tasks2 ||
     !splits || !packed || !incl || !acc || !chunk_task || !chunk_part || !bin_slot || !gbins ||
     !gcounter) {
    return false;
  }
  uint32_t hb[12];
  if(!cuda_ok(cudaMemcpyAsync(hb, d_bounds, sizeof(hb), cudaMemcpyDeviceToHost, st),
              "bounds read", err) || !cuda_ok(cudaStreamSynchronize(st), "bounds", err)) {
    return false;
  }
  k_iota<<<blocks_for(n, 256), 256, 0, st>>>(idx, n);
  if(n == 1) {
    DevBin leaf;
    for(int a = 0; a < 3; ++a) {
      leaf.lo[a] = decode_ordered(hb[a]);
      leaf.hi[a] = decode_ordered(hb[3 + a]);
    }
    leaf.left = kLeafBit;
    leaf.right = 1;
    uint32_t one = 1, zero = 0;
    if(!cuda_ok(cudaMemcpyAsync(nodes, &leaf, sizeof(leaf), cudaMemcpyHostToDevice, st), "root",
                err) ||
       !cuda_ok(cudaMemcpyAsync(count, &one, 4, cudaMemcpyHostToDevice, st), "root", err) ||
       !cuda_ok(cudaMemcpyAsync(final_idx, &zero, 4, cudaMemcpyHostToDevice, st), "root", err) ||
       !cuda_ok(cudaStreamSynchronize(st), "root", err)) {
      return false;
    }
    bt.nodes = nodes;
    bt.count = count;
    bt.leaf_idx = final_idx;
    bt.node_count = 1;
    bt.root = 0;
    return true;
  }
  Task root;
  root.node = 0;
  root.begin = 0;
  root.count = n;
  root.depth = 0;
  for(int a = 0; a < 3; ++a) {
    root.lo[a] = decode_ordered(hb[a]);
    root.hi[a] = decode_ordered(hb[3 + a]);
    root.clo[a] = decode_ordered(hb[6 + a]);
    root.chi[a] = decode_ordered(hb[9 + a]);
  }
  if(!cuda_ok(cudaMemcpyAsync(tasks, &root, sizeof(root), cudaMemcpyHostToDevice, st), "root",
              err)) {
    return false;
  }
  uint32_t T = 1, node_base = 1, levels = 0;
  while(T > 0) {
    if(++levels > kMaxSahLevels) {
      err = "internal error: binned SAH build too deep";
      return false;
    }
    k_task_chunks<<<blocks_for(T, 128), 128, 0, st>>>(tasks, T, packed);
    if(!scan_total(temp, temp_bytes, packed, incl, T, st, h_total, err)) { return false; }
    uint32_t C = uint32_t(*h_total), M = uint32_t(*h_total >> 32);
    if(C > chunk_cap || M > slot_cap) {
      err = "internal error: binned SAH chunk overflow";
      return false;
    }
    k_expand<<<blocks_for(T, 128), 128, 0, st>>>(tasks, T, packed, incl, chunk_task, chunk_part,
                                                  bin_slot, gbins, gcounter, acc);
    uint32_t cb = blocks_for(C, kWarps);
    k_bin_split<<<cb, 32 * kWarps, 0, st>>>(prim, idx, tasks, chunk_task, chunk_part, C,
                                             bin_slot, gbins, gcounter, max_leaf, splits);
    k_partition<<<cb, 32 * kWarps, 0, st>>>(prim, idx, tasks, chunk_task, chunk_part, C, splits,
                                             flags);
    size_t tb = temp_bytes;
    if(!cuda_ok(cub::DeviceScan::ExclusiveSum(temp, tb, flags, scan, int(n), st), "prefix sum",
                err)) {
      return false;
    }
    k_scatter<<<cb, 32 * kWarps, 0, st>>>(prim, idx, idx2, final_idx, tasks, chunk_task,
                                           chunk_part, C, splits, flags, scan, acc);
    k_child_counts<<<blocks_for(T, 128), 128, 0, st>>>(tasks, T, splits, packed);
    if(!scan_total(temp, temp_bytes, packed, incl, T, st, h_total, err)) { return false; }
    uint32_t made = uint32_t(*h_total), opened = uint32_t(*h_total >> 32);
    if(node_base + made > total_nodes || opened > task_cap) {
      err = "internal error: binned SAH node overflow";
      return false;
    }
    k_children<<<blocks_for(T, 128), 128, 0, st>>>(tasks, T, splits, packed, incl, acc,
                                                    node_base, nodes, count, tasks2);
    node_base += made;
    T = opened;
    std::swap(tasks, tasks2);
    std::swap(idx, idx2);
  }
  if(!cuda_ok(cudaStreamSynchronize(st), "binned SAH build", err)) { return false; }
  bt.nodes = nodes;
  bt.count = count;
  bt.leaf_idx = final_idx;
  bt.node_count = node_base;
  bt.root = 0;
  bt.iterations = levels;
  return true;
}

}  // namespace

bool build_wide_bvh_device(const float* h_verts, uint32_t vert_count, const uint32_t* h_tris,
                           uint32_t n, const BuildOptions& opts, DeviceBuilder method,
                           cudaStream_t st, DeviceBvh& out, std::string& err, BinaryDump* dump) {
  auto t0 = std::chrono::steady_clock::now();
  out = DeviceBvh();
  if(opts.max_leaf_tris < 1 || opts.max_leaf_tris > 3) {
    err = "max_leaf_tris must be 1..3";
    return false;
  }
  if(opts.width < 2 || opts.width > 8) {
    err = "bvh_width must be 2..8";
    return false;
  }
  if(n == 0) { return true; }
  if(n >= kLeafBit / 2) {
    err = "too many triangles for the device BVH build";
    return false;
  }
  Scratch sc;
  float* verts = sc.alloc<float>(3 * size_t(vert_count), err);
  uint32_t* tris = sc.alloc<uint32_t>(3 * size_t(n), err);
  DevBin* prim = sc.alloc<DevBin>(n, err);
  uint32_t* bounds = sc.alloc<uint32_t>(12, err);
  if(!verts || !tris || !prim || !bounds) { return false; }
  if(!cuda_ok(cudaMemcpyAsync(verts, h_verts, 12 * size_t(vert_count), cudaMemcpyHostToDevice,
                              st), "vertex upload", err) ||
     !cuda_ok(cudaMemcpyAsync(tris, h_tris, 12 * size_t(n), cudaMemcpyHostToDevice, st),
              "index upload", err)) {
    return false;
  }
  uint32_t binit[12];
  for(int a = 0; a < 3; ++a) {
    binit[a] = binit[6 + a] = ~0u;
    binit[3 + a] = binit[9 + a] = 0u;
  }
  if(!cuda_ok(cudaMemcpyAsync(bounds, binit, sizeof(binit), cudaMemcpyHostToDevice, st),
              "bounds init", err)) {
    return false;
  }
  k_prim_bounds<<<blocks_for(n, 256), 256, 0, st>>>(verts, tris, n, prim, bounds);

  // temporary storage for CUB, sized for the largest call
  size_t sort_bytes = 0, scan64 = 0, scan32 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<uint64_t*>(nullptr),
                                  static_cast<uint64_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), int(n), 0, 63, st);
  cub::DeviceScan::InclusiveSum(nullptr, scan64, static_cast<uint64_t*>(nullptr),
                                static_cast<uint64_t*>(nullptr), int(std::max(n, 2u)), st);
  cub::DeviceScan::ExclusiveSum(nullptr, scan32, static_cast<uint32_t*>(nullptr),
                                static_cast<uint32_t*>(nullptr), int(n), st);
  size_t temp_bytes = std::max(sort_bytes, std::max(scan64, scan32));
  void* temp = sc.alloc<unsigned char>(temp_bytes, err);
  PinnedWords pin;
  if(!temp ||
     !cuda_ok(host_pinned_alloc(&pin.p, 2 * sizeof(uint64_t)), "pinned counter", err)) {
    return false;
  }
  BinTree bt;
  if(method == DeviceBuilder::kPloc) {
    if(!build_ploc(sc, prim, bounds, n, st, temp, temp_bytes, pin.p, bt, err)) { return false; }
  } else if(!build_sah(sc, prim, bounds, n, opts.max_leaf_tris, st, temp, temp_bytes, pin.p, bt,
                       err)) {
    return false;
  }
  out.iterations = bt.iterations;

  if(dump) {
    if(!cuda_ok(cudaStreamSynchronize(st), "build", err)) { return false; }
    std::vector<DevBin> hb(bt.node_count);
    dump->count.resize(bt.node_count);
    dump->leaf_idx.resize(n);
    if(!cuda_ok(cudaMemcpy(hb.data(), bt.nodes, bt.node_count * sizeof(DevBin),
                           cudaMemcpyDeviceToHost), "tree download", err) ||
       !cuda_ok(cudaMemcpy(dump->count.data(), bt.count, bt.node_count * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost), "tree download", err) ||
       !cuda_ok(cudaMemcpy(dump->leaf_idx.data(), bt.leaf_idx, n * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost), "tree download", err)) {
      return false;
    }
    dump->lo.resize(3 * size_t(bt.node_count));
    dump->hi.resize(3 * size_t(bt.node_count));
    dump->left.resize(bt.node_count);
    dump->right.resize(bt.node_count);
    for(uint32_t i = 0; i < bt.node_count; ++i) {
      for(int a = 0; a < 3; ++a) {
        dump->lo[3 * size_t(i) + a] = hb[i].lo[a];
        dump->hi[3 * size_t(i) + a] = hb[i].hi[a];
      }
      dump->left[i] = hb[i].left;
      dump->right[i] = hb[i].right;
    }
    dump->root = bt.root;
  }

  // collapse, one level at a time
  const DevBin* nodes = bt.nodes;
  const uint32_t* count = bt.count;
  uint32_t width = std::min(8u, std::max(2u, opts.width));
  uint32_t level_cap = n / (opts.max_leaf_tris + 1) + 2;
  uint32_t* qbin = sc.alloc<uint32_t>(level_cap, err);
  uint32_t* qwide = sc.alloc<uint32_t>(level_cap, err);
  uint32_t* qbin2 = sc.alloc<uint32_t>(level_cap, err);
  uint32_t* qwide2 = sc.alloc<uint32_t>(level_cap, err);
  Plan* plans = sc.alloc<Plan>(level_cap, err);
  uint64_t* counts = sc.alloc<uint64_t>(level_cap, err);
  uint64_t* incl = sc.alloc<uint64_t>(level_cap, err);
  uint32_t* d_err = sc.alloc<uint32_t>(1, err);
  if(!qbin || !qwide || !qbin2 || !qwide2 || !plans || !counts || !incl || !d_err) {
    return false;
  }
#ifndef DORT_NODE_QUANTIZED
  constexpr bool kFloat = true;
  const size_t node_size = sizeof(WideNodeF);
#else
  constexpr bool kFloat = false;
  const size_t node_size = sizeof(WideNode);
#endif
  size_t wide_cap = std::max<size_t>(16, n / 4 + 16);
  void* wide = nullptr;
  if(dev_alloc(&wide, wide_cap * node_size) != cudaSuccess) {
    cudaGetLastError();
    err = "cudaMalloc of the BVH nodes failed";
    return false;
  }
  LeafTri* leaf = nullptr;
  if(dev_alloc(&leaf, size_t(n) * sizeof(LeafTri)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(wide);
    err = "cudaMalloc of the BVH triangles failed";
    return false;
  }
  struct Owned {
    void*& w; LeafTri*& l; bool keep = false;
    ~Owned() { if(!keep) { if(w) { cudaFree(w); } if(l) { cudaFree(l); } } }
  } owned{wide, leaf};
  uint32_t root_bin = bt.root, root_wide = 0;
  if(!cuda_ok(cudaMemcpyAsync(qbin, &root_bin, 4, cudaMemcpyHostToDevice, st), "queue", err) ||
     !cuda_ok(cudaMemcpyAsync(qwide, &root_wide, 4, cudaMemcpyHostToDevice, st), "queue", err) ||
     !cuda_ok(cudaMemsetAsync(d_err, 0, 4, st), "error flag", err)) {
    return false;
  }
  uint32_t items = 1, wide_count = 1, tri_count = 0, depth = 0;
  while(items > 0) {
    if(++depth > kMaxWideDepth) {
      err = "BVH too deep for the device traversal stack";
      return false;
    }
    k_plan<<<blocks_for(items, 128), 128, 0, st>>>(nodes, count, qbin, items, width,
                                                    opts.max_leaf_tris, plans, counts);
    if(!scan_total(temp, temp_bytes, counts, incl, items, st, pin.p, err)) { return false; }
    uint32_t children = uint32_t(*pin.p);
    uint32_t leaf_tris = uint32_t(*pin.p >> 32);
    if(children > level_cap || tri_count + leaf_tris > n) {
      err = "internal error: wide BVH level overflow";
      return false;
    }
    if(wide_count + children > wide_cap) {
      size_t cap2 = std::max<size_t>(wide_cap * 2, wide_count + children);
      void* w2 = nullptr;
      if(dev_alloc(&w2, cap2 * node_size) != cudaSuccess) {
        cudaGetLastError();
        err = "cudaMalloc of the BVH nodes failed";
        return false;
      }
      if(!cuda_ok(cudaMemcpyAsync(w2, wide, wide_count * node_size, cudaMemcpyDeviceToDevice,
                                  st), "node copy", err) ||
         !cuda_ok(cudaStreamSynchronize(st), "node copy", err)) {
        cudaFree(w2);
        return false;
      }
      cudaFree(wide);
      wide = w2;
      wide_cap = cap2;
    }
    k_emit<kFloat><<<blocks_for(items, 128), 128, 0, st>>>(
        nodes, count, bt.leaf_idx, verts, tris, qbin, qwide, items, opts.max_leaf_tris, plans,
        counts, incl, wide_count, tri_count, wide, leaf, qbin2, qwide2, d_err);
    wide_count += children;
    tri_count += leaf_tris;
    items = children;
    std::swap(qbin, qbin2);
    std::swap(qwide, qwide2);
  }
  uint32_t h_err = 0;
  if(!cuda_ok(cudaMemcpyAsync(&h_err, d_err, 4, cudaMemcpyDeviceToHost, st), "error read", err) ||
     !cuda_ok(cudaStreamSynchronize(st), "collapse", err)) {
    return false;
  }
  if(h_err & 1u) {
    err = "BVH quantization failed (scene coordinates out of range)";
    return false;
  }
  if(h_err || tri_count != n) {
    err = "internal error: wide BVH leaf overflow";
    return false;
  }
  owned.keep = true;
  out.nodes = wide;
  out.node_bytes = wide_cap * node_size;
  out.node_count = wide_count;
  out.tris = leaf;
  out.tri_count = tri_count;
  out.depth = depth;
  out.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
               .count();
  return true;
}

}  // namespace dort_gpu

// ---- diagnostics ----------------------------------------------------------------

using namespace dort_gpu;

extern "C" int dort_gpu_scene_bvh_cost(const dort_scene* s, double out[4]) try {
  clear_error();
  if(!s || !out) { return fail(DORT_ERR_INVALID, "null argument"); }
  size_t count = s->trace.node_count;
  std::vector<WideNodeF> f(count);
#ifndef DORT_NODE_QUANTIZED
  if(count) {
    DG_CUDA(cudaMemcpy(f.data(), s->trace.nodes, count * sizeof(WideNodeF),
                       cudaMemcpyDeviceToHost));
  }
#else
  std::vector<WideNode> q(count);
  if(count) {
    DG_CUDA(cudaMemcpy(q.data(), s->trace.nodes, count * sizeof(WideNode),
                       cudaMemcpyDeviceToHost));
  }
  expand_node_planes(q, f);
#endif
  size_t leaf_slots = 0;
  for(const WideNodeF& n : f) {
    for(int k = 0; k < 8; ++k) {
      if(n.meta[k] != 0 && !(n.imask & (1u << k))) { ++leaf_slots; }
    }
  }
  out[0] = wide_sah_cost(f.data(), f.size());
  out[1] = double(count);
  out[2] = double(leaf_slots);
  out[3] = s->depth;
  return DORT_OK;
} DORT_ABI_CATCH

extern "C" int dort_gpu_check_device_bvh(const dort_scene_desc* desc, double out[8]) try {
  clear_error();
  if(!desc || !out) { return fail(DORT_ERR_INVALID, "null argument"); }
  if(desc->struct_size != sizeof(dort_scene_desc)) {
    return fail(DORT_ERR_INVALID, "dort_scene_desc.struct_size mismatch (ABI version)");
  }
  std::string err;
  if(!validate_mesh(desc->verts, desc->vert_count, desc->tris, desc->tri_count, err)) {
    return fail(DORT_ERR_INVALID, err);
  }
  BuildOptions opts;
  opts.width = desc->bvh_width ? desc->bvh_width : 8;
  DeviceBvh db;
  BinaryDump dump;
  DeviceBuilder method =
      desc->bvh_build == DORT_BVH_BUILD_PLOC ? DeviceBuilder::kPloc : DeviceBuilder::kSah;
  if(!build_wide_bvh_device(desc->verts, desc->vert_count, desc->tris, desc->tri_count, opts,
                            method, nullptr, db, err, &dump)) {
    return fail(DORT_ERR_CUDA, err);
  }
  struct Free {
    DeviceBvh& b;
    ~Free() { if(b.nodes) { cudaFree(b.nodes); } if(b.tris) { cudaFree(b.tris); } }
  } fr{db};
  WideBvh host;
  if(!collapse_binary_dump(dump, desc->verts, desc->tris, desc->tri_count, opts, host, err)) {
    return fail(DORT_ERR_INVALID, err);
  }
  const unsigned char* hn = static_cast<const unsigned char*>(traversal_nodes(host));
  size_t hn_bytes = traversal_node_bytes(host);
  size_t node_size = db.node_count ? hn_bytes / std::max<size_t>(host.nodes.size(), 1) : 0;
  std::vector<unsigned char> dn(size_t(db.node_count) * node_size);
  std::vector<LeafTri> dt(db.tri_count);
  if(!dn.empty()) { DG_CUDA(cudaMemcpy(dn.data(), db.nodes, dn.size(), cudaMemcpyDeviceToHost)); }
  if(!dt.empty()) {
    DG_CUDA(cudaMemcpy(dt.data(), db.tris, dt.size() * sizeof(LeafTri), cudaMemcpyDeviceToHost));
  }
  double node_diff = 0, tri_diff = 0;
  if(dn.size() != hn_bytes) {
    node_diff = double(std::max(dn.size(), hn_bytes));
  } else {
    for(size_t i = 0; i < hn_bytes; ++i) { node_diff += dn[i] != hn[i]; }
  }
  const unsigned char* ht = reinterpret_cast<const unsigned char*>(host.tris.data());
  const unsigned char* dtb = reinterpret_cast<const unsigned char*>(dt.data());
  size_t tb = dt.size() * sizeof(LeafTri);
  if(host.tris.size() != dt.size()) {
    tri_diff = double(std::max(host.tris.size(), dt.size()) * sizeof(LeafTri));
  } else {
    for(size_t i = 0; i < tb; ++i) { tri_diff += dtb[i] != ht[i]; }
  }
  std::vector<uint32_t> seen(desc->tri_count, 0);
  bool once = dt.size() == desc->tri_count;
  for(const LeafTri& t : dt) {
    if(t.id >= desc->tri_count || seen[t.id]++) { once = false; }
  }
  std::vector<WideNodeF> f;
#ifndef DORT_NODE_QUANTIZED
  f.resize(db.node_count);
  if(!f.empty()) { std::memcpy(f.data(), dn.data(), dn.size()); }
#else
  std::vector<WideNode> q(db.node_count);
  if(!q.empty()) { std::memcpy(q.data(), dn.data(), dn.size()); }
  expand_node_planes(q, f);
#endif
  out[0] = node_diff;
  out[1] = tri_diff;
  out[2] = db.node_count;
  out[3] = once ? 1.0 : 0.0;
  out[4] = db.ms;
  out[5] = db.iterations;
  out[6] = db.depth;
  out[7] = wide_sah_cost(f.data(), f.size());
  return DORT_OK;
} DORT_ABI_CATCH
