"""ctypes view of the C ABI in include/dort_gpu.h.

Loads the in-tree ``libdort_gpu.so``.  There is no fallback: if the library
is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
# DORT_GPU_LIBRARY selects another build of the same library (e.g. an
# installed copy); the default is the in-tree build.
LIB_PATH = os.environ.get("DORT_GPU_LIBRARY") or os.path.join(PKG, "libdort_gpu.so")

c_u32 = ctypes.c_uint32
c_i32 = ctypes.c_int
c_size = ctypes.c_size_t
c_f = ctypes.c_float
c_p = ctypes.c_void_p

DORT_OK = 0
STATUS_NAMES = {
    0: "DORT_OK", -1: "DORT_ERR_INVALID", -2: "DORT_ERR_CUDA", -3: "DORT_ERR_OOM",
    -4: "DORT_ERR_TIMEOUT", -5: "DORT_ERR_UNSUPPORTED", -6: "DORT_ERR_DEVICE",
}
MISS = 0xFFFFFFFF

MAT_LAMBERT, MAT_MIRROR, MAT_DIELECTRIC, MAT_PHONG, MAT_CONDUCTOR, MAT_OREN_NAYAR = range(6)
SHAPE_SPHERE, SHAPE_DISK, SHAPE_CUBE, SHAPE_CYLINDER = 1, 2, 3, 4
SHAPE_LIGHT_TRANSFORM = 1
LIGHT_POINT, LIGHT_DIRECTIONAL = 1, 2
CAMERA_PINHOLE, CAMERA_ORTHO, CAMERA_THIN_LENS = 0, 1, 2
BVH_BUILD_DEFAULT, BVH_BUILD_HOST, BVH_BUILD_DEVICE, BVH_BUILD_PLOC = 0, 1, 2, 3
RENDERER_PT, RENDERER_LT, RENDERER_BDPT = 0, 1, 2
BDPT_NO_T1_PATHS = 1
PT_NO_ROULETTE = 2
ADJOINT_MEGAKERNEL = 4
SCENE_WATERTIGHT = 1
ABI_VERSION = 2


class Material(ctypes.Structure):
    _fields_ = [("kind", c_u32), ("color", c_f * 3), ("color2", c_f * 3),
                ("param", c_f * 4)]


class Shape(ctypes.Structure):
    _fields_ = [("kind", c_u32), ("material", c_u32), ("param", c_f * 4),
                ("to_world", c_f * 12), ("emission", c_f * 3), ("flags", c_u32),
                ("light_to_world", c_f * 12)]


class Light(ctypes.Structure):
    _fields_ = [("kind", c_u32), ("rgb", c_f * 3), ("vec", c_f * 3), ("reserved", c_u32)]


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", c_u32),
        ("verts", c_p), ("vert_count", c_u32),
        ("tris", c_p), ("tri_count", c_u32),
        ("tri_material", c_p),
        ("materials", c_p), ("material_count", c_u32),
        ("tri_emission", c_p),
        ("sky_rgb", c_p), ("sky_width", c_u32), ("sky_height", c_u32),
        ("sky_const", c_f * 3),
        ("sky_scale", c_f * 3),
        ("sky_up", c_f * 3),
        ("sky_fwd", c_f * 3),
        ("bvh_width", c_u32),
        ("shape_count", c_u32),
        ("shapes", c_p),
        ("lights", c_p),
        ("light_count", c_u32),
        ("bvh_build", c_u32),
        ("tri_light_verts", c_p),
        ("flags", c_u32),
        ("reserved", c_u32 * 1),
    ]


class Camera(ctypes.Structure):
    _fields_ = [("origin", c_f * 3), ("right", c_f * 3), ("up", c_f * 3),
                ("forward", c_f * 3), ("fov", c_f), ("kind", c_u32),
                ("lens_radius", c_f), ("focal_distance", c_f), ("dimension", c_f)]


class RenderParams(ctypes.Structure):
    _fields_ = [
        ("struct_size", c_u32), ("width", c_u32), ("height", c_u32),
        ("iterations", c_u32), ("min_depth", c_u32), ("max_depth", c_u32),
        ("only_direct", c_u32), ("sample_all_lights", c_u32),
        ("direct_strategy", c_u32), ("renderer", c_u32), ("seed", ctypes.c_uint64),
        ("camera", Camera), ("renderer_flags", c_u32), ("reserved", c_u32 * 7),
    ]


class WavefrontTuning(ctypes.Structure):
    _fields_ = [("struct_size", c_u32), ("queue_capacity", c_u32), ("trace_block", c_u32),
                ("shade_block", c_u32), ("sort_rays", c_u32), ("max_waves", c_u32),
                ("stage_queues", c_u32), ("deterministic", c_u32)]


class BatchJob(ctypes.Structure):
    _fields_ = [("scene", c_p), ("params", RenderParams)]


class DortError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m dort_b200.build` "
                "(the CUDA library is required; there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.dort_gpu_last_error.restype = ctypes.c_char_p
        L.dort_gpu_last_error.argtypes = []
        L.dort_gpu_abi_version.restype = c_i32
        if L.dort_gpu_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {L.dort_gpu_abi_version()}, "
                               f"expected {ABI_VERSION}: rebuild it")
        L.dort_gpu_scene_create.restype = c_i32
        L.dort_gpu_scene_create.argtypes = [ctypes.POINTER(SceneDesc), ctypes.POINTER(c_p)]
        L.dort_gpu_scene_destroy.restype = c_i32
        L.dort_gpu_scene_destroy.argtypes = [c_p]
        L.dort_gpu_scene_stats.restype = c_i32
        L.dort_gpu_scene_stats.argtypes = [c_p, ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_raycast.restype = c_i32
        L.dort_gpu_raycast.argtypes = [c_p, c_p, c_size, c_i32, c_p, c_p]
        L.dort_gpu_raycast_device.restype = c_i32
        L.dort_gpu_raycast_device.argtypes = [c_p, c_p, c_size, c_i32, c_p, c_p, c_p]
        L.dort_gpu_raycast_timed.restype = c_i32
        L.dort_gpu_raycast_timed.argtypes = [c_p, c_p, c_size, c_i32, c_p, c_p, c_p,
                                             c_i32, ctypes.POINTER(c_f)]
        L.dort_gpu_host_check_raycast.restype = c_i32
        L.dort_gpu_host_check_raycast.argtypes = [ctypes.POINTER(SceneDesc), c_p, c_size,
                                                  c_i32, c_p, c_p, ctypes.POINTER(c_u32)]
        L.dort_gpu_render.restype = c_i32
        L.dort_gpu_render.argtypes = [c_p, ctypes.POINTER(RenderParams), c_p,
                                      ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_render_device.restype = c_i32
        L.dort_gpu_render_device.argtypes = [c_p, ctypes.POINTER(RenderParams), c_p, c_p]
        L.dort_gpu_host_check_render.restype = c_i32
        L.dort_gpu_host_check_render.argtypes = [ctypes.POINTER(SceneDesc),
                                                 ctypes.POINTER(RenderParams), c_u32, c_u32,
                                                 c_p]
        L.dort_gpu_render_wavefront.restype = c_i32
        L.dort_gpu_render_wavefront.argtypes = [c_p, ctypes.POINTER(RenderParams),
                                                ctypes.POINTER(WavefrontTuning), c_p,
                                                ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_render_wavefront_device.restype = c_i32
        L.dort_gpu_render_wavefront_device.argtypes = [c_p, ctypes.POINTER(RenderParams),
                                                       ctypes.POINTER(WavefrontTuning), c_p, c_p]
        L.dort_gpu_wavefront_stage_times.restype = c_i32
        L.dort_gpu_wavefront_stage_times.argtypes = [c_p, ctypes.POINTER(RenderParams),
                                                     ctypes.POINTER(WavefrontTuning),
                                                     ctypes.POINTER(ctypes.c_double),
                                                     ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_adjoint_forward.restype = c_i32
        L.dort_gpu_adjoint_forward.argtypes = [c_p, ctypes.POINTER(RenderParams), c_p, c_p, c_p]
        L.dort_gpu_adjoint_backward.restype = c_i32
        L.dort_gpu_adjoint_backward.argtypes = [c_p, ctypes.POINTER(RenderParams), c_p, c_p, c_p,
                                                c_p, c_p]
        L.dort_gpu_debug_adjoint_list.restype = c_i32
        L.dort_gpu_debug_adjoint_list.argtypes = [ctypes.c_longlong]
        L.dort_gpu_adjoint_stats.restype = c_i32
        L.dort_gpu_adjoint_stats.argtypes = [c_p, ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_loss_l2.restype = c_i32
        L.dort_gpu_loss_l2.argtypes = [c_p, c_p, c_size, ctypes.POINTER(ctypes.c_double), c_p]
        L.dort_gpu_render_device_noalloc.restype = c_i32
        L.dort_gpu_render_device_noalloc.argtypes = [c_p, ctypes.POINTER(RenderParams), c_p,
                                                     c_p]
        L.dort_gpu_batch_create.restype = c_i32
        L.dort_gpu_batch_create.argtypes = [ctypes.POINTER(BatchJob), c_u32,
                                            ctypes.POINTER(WavefrontTuning), ctypes.POINTER(c_p)]
        L.dort_gpu_batch_render.restype = c_i32
        L.dort_gpu_batch_render.argtypes = [c_p, c_p]
        L.dort_gpu_batch_image.restype = c_i32
        L.dort_gpu_batch_image.argtypes = [c_p, c_u32, c_p]
        L.dort_gpu_batch_image_device.restype = c_i32
        L.dort_gpu_batch_image_device.argtypes = [c_p, c_u32, ctypes.POINTER(c_p)]
        L.dort_gpu_batch_stats.restype = c_i32
        L.dort_gpu_batch_stats.argtypes = [c_p, ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_batch_destroy.restype = c_i32
        L.dort_gpu_batch_destroy.argtypes = [c_p]
        L.dort_gpu_scene_bvh_cost.restype = c_i32
        L.dort_gpu_scene_bvh_cost.argtypes = [c_p, ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_bsdf_probe.restype = c_i32
        L.dort_gpu_bsdf_probe.argtypes = [ctypes.POINTER(Material), c_size, c_p, c_p, c_p, c_p,
                                          c_p, c_p, c_p, c_p, c_i32]
        L.dort_gpu_autotune_wavefront.restype = c_i32
        L.dort_gpu_autotune_wavefront.argtypes = [c_p, ctypes.POINTER(RenderParams),
                                                  ctypes.c_double, ctypes.POINTER(WavefrontTuning),
                                                  ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_autotune_batch.restype = c_i32
        L.dort_gpu_autotune_batch.argtypes = [ctypes.POINTER(BatchJob), c_u32, ctypes.c_double,
                                              ctypes.POINTER(WavefrontTuning),
                                              ctypes.POINTER(ctypes.c_double)]
        L.dort_gpu_debug_fail_alloc.restype = c_i32
        L.dort_gpu_debug_fail_alloc.argtypes = [ctypes.c_longlong]
        L.dort_gpu_check_device_bvh.restype = c_i32
        L.dort_gpu_check_device_bvh.argtypes = [ctypes.POINTER(SceneDesc),
                                                ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != DORT_OK:
        msg = lib().dort_gpu_last_error().decode(errors="replace")
        raise DortError(status, msg)
