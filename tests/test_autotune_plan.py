"""CPU checks of the wavefront's path-slot rules (dort_b200/csrc/autotune_plan.h):
which capacities the queue allocation accepts and which the autotuner tries.

The header is plain C++; the test compiles it with g++ into a small shared
object, so the cases that only large GPUs or many-light scenes reach (2^28
slots, every light sampled, little free memory) run without a GPU.
"""
import ctypes
import shutil
import subprocess
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dort_b200", "csrc")

SHIM = r'''
#include "autotune_plan.h"
extern "C" double slot_bytes(unsigned nee) { return dort_gpu::wavefront_slot_bytes(nee); }
extern "C" int entries_fit(unsigned cap, unsigned nee) {
  return dort_gpu::wavefront_entries_fit(cap, nee) ? 1 : 0;
}
extern "C" int candidate(unsigned cap, int first, unsigned long long units, unsigned nee,
                         unsigned long long free_bytes, unsigned held) {
  return dort_gpu::capacity_candidate(cap, first != 0, units, nee, size_t(free_bytes), held)
      ? 1 : 0;
}
'''

GB = 1 << 30


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("autotune_plan")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    so = d / "libautotune_plan.so"
    subprocess.run([gxx, "-std=c++17", "-O1", "-shared", "-fPIC", "-I" + CSRC, str(src), "-o",
                    str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.slot_bytes.restype = ctypes.c_double
    lib.slot_bytes.argtypes = [ctypes.c_uint]
    lib.entries_fit.argtypes = [ctypes.c_uint, ctypes.c_uint]
    lib.candidate.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_uint,
                              ctypes.c_ulonglong, ctypes.c_uint]
    return lib


def test_slot_bytes(lib):
    # one light per vertex: the 340 bytes a slot takes in the frame's queues
    assert lib.slot_bytes(1) == 340.0
    assert lib.slot_bytes(8) == 184.0 + 8 * 156.0


def test_entry_counters(lib):
    assert lib.entries_fit(1 << 28, 1) == 1
    assert lib.entries_fit(1 << 28, 4) == 1
    assert lib.entries_fit(1 << 28, 5) == 0
    assert lib.entries_fit(1 << 26, 16) == 1
    assert lib.entries_fit(1 << 26, 17) == 0


def test_frame_candidates(lib):
    units_1080p = 1920 * 1080 * 256      # one-sample units of the 1080p frame
    free = 178 * GB
    # one light per vertex: every capacity up to 2^28 on a B200's free memory
    for k in range(22, 29):
        assert lib.candidate(1 << k, 0, units_1080p, 1, free, 1 << 22) == 1
    # every light sampled with 8 lights: 2^28 breaks the counters, 2^27 the
    # memory (1,432 bytes per slot), 2^26 fits
    assert lib.candidate(1 << 28, 0, units_1080p, 8, free, 0) == 0
    assert lib.candidate(1 << 27, 0, units_1080p, 8, free, 0) == 0
    assert lib.candidate(1 << 26, 0, units_1080p, 8, free, 0) == 1
    # a small frame: nothing above twice its units, but the first candidate
    # always
    assert lib.candidate(1 << 23, 0, 1 << 20, 1, free, 0) == 0
    assert lib.candidate(1 << 22, 1, 1 << 20, 1, free, 0) == 1


def test_held_queues_count_as_free(lib):
    """The scene's current queues are released before the next capacity is
    allocated, so their bytes count as available."""
    held = 1 << 26                        # 21.25 GB of queues
    free = int(40 * GB)                   # 2^27 slots need 42.5 GB
    assert lib.candidate(1 << 27, 0, 1 << 30, 1, free, 0) == 0
    assert lib.candidate(1 << 27, 0, 1 << 30, 1, free, held) == 1
