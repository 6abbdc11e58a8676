// Which path-slot capacities the wavefront can take and the autotuner tries.
// Plain host C++ (no CUDA types), so the rules can be checked on a machine
// without a GPU.
//
// A path slot holds about 184 bytes of path state, queues and sort buffers,
// plus 156 bytes of direct-lighting queues per light a vertex samples
// (nee_mult: the light count when every light is sampled, else 1): two
// shadow entries (slot index, origin, direction, contribution) and one
// BSDF-strategy entry per light, wavefront.cu (wf_alloc).  The queues'
// entries of one wave are counted in 32 bits.
#pragma once
#include <cstddef>
#include <cstdint>

namespace dort_gpu {

inline double wavefront_slot_bytes(uint32_t nee_mult) {
  return 184.0 + 156.0 * double(nee_mult);
}

// The direct-lighting queues of `capacity` slots stay within their 32-bit
// counters: 2 * nee_mult * capacity <= 2^31.
inline bool wavefront_entries_fit(uint32_t capacity, uint32_t nee_mult) {
  return 2ull * nee_mult * capacity <= (1ull << 31);
}

// Whether the autotuner's capacity step times `cap` slots for a frame of
// `units` work units: the first candidate always (clamped to the units by the
// caller); the others when not above twice the units, within the counters,
// and within 80 % of the free device memory plus what the scene's queues
// already hold (`held` slots, freed when the queues are reallocated).
inline bool capacity_candidate(uint32_t cap, bool first, uint64_t units, uint32_t nee_mult,
                               size_t free_bytes, uint32_t held) {
  if(first) { return true; }
  if(uint64_t(cap) > 2 * units) { return false; }
  if(!wavefront_entries_fit(cap, nee_mult)) { return false; }
  const double have = double(free_bytes) + wavefront_slot_bytes(nee_mult) * double(held);
  return wavefront_slot_bytes(nee_mult) * double(cap) <= 0.8 * have;
}

}  // namespace dort_gpu
