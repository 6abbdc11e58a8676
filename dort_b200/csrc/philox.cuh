// Philox4x32-10 counter-based random numbers (Salmon, Moraes, Dror, Shaw,
// "Parallel Random Numbers: As Easy as 1, 2, 3", SC 2011).
//
// The reference draws its samples from one std::mt19937 per tile
// (include/dort/rng.hpp:6-28), so its sequences depend on thread scheduling.
// Here every sample dimension is a pure function of (seed, pixel, sample,
// dimension block): paths can be regenerated exactly (path replay in the
// adjoint) and results do not depend on the launch shape.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define PHILOX_HD __host__ __device__ __forceinline__
#else
#define PHILOX_HD inline
#endif

namespace dort_gpu {

struct U4 { uint32_t x, y, z, w; };

PHILOX_HD void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
  hi = __umulhi(a, b);
  lo = a * b;
#else
  uint64_t p = uint64_t(a) * uint64_t(b);
  hi = uint32_t(p >> 32);
  lo = uint32_t(p);
#endif
}

// Ten rounds of the Philox-4x32 bijection keyed by (k0, k1).
PHILOX_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for(int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    philox_mulhilo(M0, c.x, hi0, lo0);
    philox_mulhilo(M1, c.z, hi1, lo1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// 24-bit uniform float in [0, 1).
PHILOX_HD float u01(uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }

// Four uniforms of dimension block `block` of sample `sample` of pixel
// `pixel` for the stream keyed by `seed`.
struct Rand4 { float a, b, c, d; };

PHILOX_HD Rand4 rand4(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t block) {
  U4 c = {pixel, sample, block, 0x64307274u};
  U4 r = philox4x32_10(c, uint32_t(seed), uint32_t(seed >> 32));
  return {u01(r.x), u01(r.y), u01(r.z), u01(r.w)};
}

// Dimension-block layout of one path sample.
//   block 0                  camera jitter (a, b)
//   block 1 + 3*b + {0,1,2}  bounce b: light pick, BSDF-strategy direct
//                            sample (uv, component), light sample (uv),
//                            continuation sample (uv, component), roulette
//   block 4096 + 2*(b*L + l) sample_all_lights: per light l at bounce b
constexpr uint32_t kBlockCamera = 0;
PHILOX_HD uint32_t bounce_block(uint32_t bounce) { return 1u + 3u * bounce; }
PHILOX_HD uint32_t all_lights_block(uint32_t bounce, uint32_t light, uint32_t light_count) {
  return 4096u + 2u * (bounce * light_count + light);
}

}  // namespace dort_gpu
