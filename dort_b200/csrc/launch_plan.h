// Launch shape of the per-pixel megakernel: how many sample slices run side
// by side, and the checks made before any kernel is launched.  Plain host
// C++ (no CUDA types), so the choice can be checked on a machine without a
// GPU.
//
// A slice is a contiguous range of a pixel's samples run by one thread; the
// partial sums of every (slice, pixel) pair are kept in scratch memory and a
// resolve step adds them.  The slice count aims at about four waves of 1024
// threads per SM; with a scratch of fixed size (the no-allocation entry
// point) it is further capped so that slices * pixels partial sums fit.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>

namespace dort_gpu {

struct MegaPlan {
  uint32_t slices = 0;      // sample slices per pixel
  uint32_t per = 0;         // samples per slice (the last slice may be short)
  uint32_t per_slice = 0;   // threads per slice: whole 8x4 pixel tiles
  const char* why = "";     // reason when the plan is refused
};

// Returns 0 with *out filled, or a negative dort_status with out->why set:
//   -1 (DORT_ERR_INVALID) when the scene lives on another device than the
//      current one (its BVH and triangle pointers are that device's memory),
//      or when the image needs more partial sums than max_pixels.
// max_pixels = 0 means the scratch grows to fit (no cap).
inline int megakernel_plan(int scene_device, int current_device, int sms, uint32_t width,
                           uint32_t height, uint32_t spp, size_t max_pixels, MegaPlan* out) {
  if(scene_device != current_device) {
    out->why = "scene on another device than the current one";
    return -1;
  }
  const uint64_t npix = uint64_t(width) * height;
  if(npix == 0 || spp == 0) {
    out->why = "empty image";
    return -1;
  }
  if(max_pixels != 0 && npix > max_pixels) {
    out->why = "image exceeds the scratch limit";
    return -1;
  }
  const uint64_t target = uint64_t(std::max(sms, 1)) * 1024 * 4;
  uint64_t slices = std::min<uint64_t>(spp, std::max<uint64_t>(1, target / npix));
  if(max_pixels != 0) {
    slices = std::min<uint64_t>(slices, std::max<uint64_t>(1, max_pixels / npix));
  }
  const uint64_t per = (spp + slices - 1) / slices;
  slices = (spp + per - 1) / per;
  out->slices = uint32_t(slices);
  out->per = uint32_t(per);
  out->per_slice = uint32_t(uint64_t((width + 7) / 8) * ((height + 3) / 4) * 32);
  return 0;
}

}  // namespace dort_gpu
