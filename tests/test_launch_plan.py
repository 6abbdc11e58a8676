"""CPU checks of the megakernel's launch plan (dort_b200/csrc/launch_plan.h):
the checks every per-pixel render makes before it launches anything, and the
slice count, including the cap that keeps the no-allocation entry point's
partial sums inside its fixed scratch.

The header is plain C++; the test compiles it with g++ into a small shared
object, so these cases run without a GPU -- in particular the scene-on-another
device refusal, which a one-GPU machine cannot produce with real scenes.
"""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dort_b200", "csrc")

SHIM = r'''
#include "launch_plan.h"
extern "C" int plan(int scene_dev, int cur_dev, int sms, unsigned w, unsigned h, unsigned spp,
                    unsigned long long max_pixels, unsigned* out) {
  dort_gpu::MegaPlan p;
  int rc = dort_gpu::megakernel_plan(scene_dev, cur_dev, sms, w, h, spp, size_t(max_pixels), &p);
  out[0] = p.slices; out[1] = p.per; out[2] = p.per_slice;
  return rc;
}
'''

# the no-allocation entry point's scratch: 16 MiB less a 256-byte header, in
# 16-byte partial sums (render_noalloc.cu)
NOALLOC_MAX_PIXELS = ((16 << 20) - 256) // 16


@pytest.fixture(scope="module")
def plan(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("plan")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    so = d / "libplan.so"
    subprocess.run([gxx, "-std=c++17", "-O1", "-shared", "-fPIC", "-I" + CSRC, str(src), "-o",
                    str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.plan.restype = ctypes.c_int
    lib.plan.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint,
                         ctypes.c_uint, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_uint)]

    def call(scene_dev, cur_dev, sms, w, h, spp, max_pixels=0):
        out = (ctypes.c_uint * 3)()
        rc = lib.plan(scene_dev, cur_dev, sms, w, h, spp, max_pixels, out)
        return rc, tuple(out)
    return call


def test_scene_on_another_device_is_refused(plan):
    rc, _ = plan(1, 0, 148, 64, 64, 16)
    assert rc == -1
    rc, _ = plan(0, 3, 148, 64, 64, 16, NOALLOC_MAX_PIXELS)
    assert rc == -1
    rc, (slices, per, per_slice) = plan(2, 2, 148, 64, 64, 16)
    assert rc == 0 and slices * per >= 16


def test_slices_cover_every_sample_once(plan):
    for (w, h, spp) in ((1, 1, 1), (7, 3, 5), (96, 64, 16), (1920, 1080, 256), (512, 512, 64),
                        (33, 17, 1000)):
        rc, (slices, per, per_slice) = plan(0, 0, 148, w, h, spp)
        assert rc == 0
        assert (slices - 1) * per < spp <= slices * per
        assert per_slice == ((w + 7) // 8) * ((h + 3) // 4) * 32


def test_noalloc_cap_keeps_partial_sums_inside_the_scratch(plan):
    # a GPU with many SMs asks for more slices than the scratch holds: the
    # cap must bring slices * pixels back under the limit
    for sms in (148, 4096, 1 << 16):
        for (w, h, spp) in ((16, 16, 4096), (64, 64, 1024), (100, 100, 300), (1020, 1024, 16),
                            (1, 1, 1 << 20)):
            rc, (slices, per, _) = plan(0, 0, sms, w, h, spp, NOALLOC_MAX_PIXELS)
            assert rc == 0
            assert slices * w * h <= NOALLOC_MAX_PIXELS
            assert (slices - 1) * per < spp <= slices * per
    # with 2^16 SMs the uncapped plan would exceed the scratch: the cap is live
    rc, (slices, _, _) = plan(0, 0, 1 << 16, 64, 64, 1024)
    assert rc == 0 and slices * 64 * 64 > NOALLOC_MAX_PIXELS
    rc, (slices, _, _) = plan(0, 0, 1 << 16, 64, 64, 1024, NOALLOC_MAX_PIXELS)
    assert rc == 0 and slices * 64 * 64 <= NOALLOC_MAX_PIXELS


def test_images_beyond_the_scratch_are_refused(plan):
    rc, _ = plan(0, 0, 148, 1024, 1024, 1, NOALLOC_MAX_PIXELS)   # 1,048,576 pixels
    assert rc == -1
    rc, _ = plan(0, 0, 148, 1020, 1028, 1, NOALLOC_MAX_PIXELS)   # 1,048,560 pixels
    assert rc == 0
