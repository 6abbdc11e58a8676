"""dort_b200 -- B200-native (sm_100a) path-tracing hot path of the dort renderer.

Python host mirror of the C ABI in ``include/dort_gpu.h``.  Every call goes
through the CUDA library ``libdort_gpu.so`` built in-tree; nothing here
computes a ray query or a render on the CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import (CAMERA_ORTHO, CAMERA_PINHOLE, CAMERA_THIN_LENS, DortError, LIGHT_DIRECTIONAL,
                   LIGHT_POINT, MISS, MAT_CONDUCTOR, MAT_DIELECTRIC, MAT_LAMBERT, MAT_MIRROR,
                   MAT_OREN_NAYAR, MAT_PHONG, SHAPE_CUBE, SHAPE_CYLINDER, SHAPE_DISK,
                   SHAPE_SPHERE)

__all__ = ["Scene", "DortError", "MISS", "host_check_raycast", "scene_desc", "check_device_bvh",
           "MAT_LAMBERT", "MAT_MIRROR", "MAT_DIELECTRIC", "MAT_PHONG", "MAT_CONDUCTOR",
           "MAT_OREN_NAYAR", "SHAPE_SPHERE", "SHAPE_DISK", "SHAPE_CUBE", "SHAPE_CYLINDER",
           "LIGHT_POINT", "LIGHT_DIRECTIONAL", "CAMERA_PINHOLE", "CAMERA_ORTHO",
           "CAMERA_THIN_LENS"]

# optional scene-dict keys passed through to scene_desc
SCENE_KEYS = ("tri_material", "materials", "tri_emission", "sky_rgb", "sky_const",
              "sky_scale", "sky_up", "sky_fwd", "shapes", "delta_lights", "tri_light_verts",
              "bvh_build", "watertight")

_BVH_BUILD = {None: _abi.BVH_BUILD_DEFAULT, "default": _abi.BVH_BUILD_DEFAULT,
              "host": _abi.BVH_BUILD_HOST, "device": _abi.BVH_BUILD_DEVICE,
              "ploc": _abi.BVH_BUILD_PLOC}


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class _DescHolder:
    """Keeps the numpy arrays a SceneDesc points to alive."""

    def __init__(self):
        self.keep = []
        self.desc = _abi.SceneDesc()

    def arr(self, a, dtype):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype)
        self.keep.append(a)
        return ctypes.c_void_p(a.ctypes.data)


def scene_desc(verts, tris, tri_material=None, materials=None, tri_emission=None,
               sky_rgb=None, sky_const=(0.0, 0.0, 0.0), sky_scale=(0.0, 0.0, 0.0),
               sky_up=(0.0, 0.0, 0.0), sky_fwd=(0.0, 0.0, 0.0),
               bvh_width: int = 8, shapes=None, delta_lights=None, tri_light_verts=None,
               bvh_build: str | None = None, watertight: bool = False,
               **_ignored) -> _DescHolder:
    """SceneDesc for the arrays given.  `shapes`: dicts with kind (SHAPE_*),
    material, param (up to 4), to_world (3x4), emission (RGB) and optionally
    light_to_world (3x4); `delta_lights`: dicts with kind (LIGHT_POINT /
    LIGHT_DIRECTIONAL), rgb and vec; `bvh_build`: "host" (binned SAH on the
    host), "device" (the same on the device), "ploc" (Morton order + PLOC on
    the device: fastest build, slower traversal) or None (the library's
    default, "device"); `watertight`: hits by the watertight ray/triangle test
    (DORT_SCENE_WATERTIGHT) instead of the reference's Moller-Trumbore."""
    h = _DescHolder()
    d = h.desc
    verts = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    tris = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    d.struct_size = ctypes.sizeof(_abi.SceneDesc)
    d.verts = h.arr(verts, np.float32)
    d.vert_count = len(verts)
    d.tris = h.arr(tris, np.uint32)
    d.tri_count = len(tris)
    d.tri_material = h.arr(tri_material, np.uint32)
    if materials:
        mats = (_abi.Material * len(materials))()
        for i, m in enumerate(materials):
            mats[i].kind = m.get("kind", MAT_LAMBERT)
            mats[i].color = (ctypes.c_float * 3)(*m.get("color", (0.0, 0.0, 0.0)))
            mats[i].color2 = (ctypes.c_float * 3)(*m.get("color2", (0.0, 0.0, 0.0)))
            p = list(m.get("param", ())) + [0.0] * 4
            mats[i].param = (ctypes.c_float * 4)(*p[:4])
        h.keep.append(mats)
        d.materials = ctypes.cast(mats, ctypes.c_void_p)
        d.material_count = len(materials)
    d.tri_emission = h.arr(tri_emission, np.float32)
    d.tri_light_verts = h.arr(tri_light_verts, np.float32)
    if sky_rgb is not None:
        sky = np.ascontiguousarray(sky_rgb, np.float32)
        d.sky_rgb = h.arr(sky, np.float32)
        d.sky_height, d.sky_width = sky.shape[0], sky.shape[1]
    d.sky_const = (ctypes.c_float * 3)(*sky_const)
    d.sky_scale = (ctypes.c_float * 3)(*sky_scale)
    d.sky_up = (ctypes.c_float * 3)(*sky_up)
    d.sky_fwd = (ctypes.c_float * 3)(*sky_fwd)
    d.bvh_width = bvh_width
    if bvh_build not in _BVH_BUILD:
        raise ValueError(f"bvh_build must be one of {sorted(k for k in _BVH_BUILD if k)}")
    d.bvh_build = _BVH_BUILD[bvh_build]
    d.flags = _abi.SCENE_WATERTIGHT if watertight else 0
    if shapes:
        arr = (_abi.Shape * len(shapes))()
        for i, sh in enumerate(shapes):
            arr[i].kind = sh["kind"]
            arr[i].material = sh.get("material", 0)
            p = list(sh.get("param", ())) + [0.0] * 4
            arr[i].param = (ctypes.c_float * 4)(*p[:4])
            m = np.asarray(sh.get("to_world", np.eye(4)[:3]), np.float64).reshape(-1)[:12]
            arr[i].to_world = (ctypes.c_float * 12)(*m.tolist())
            arr[i].emission = (ctypes.c_float * 3)(*sh.get("emission", (0.0, 0.0, 0.0)))
            if sh.get("light_to_world") is not None:
                lm = np.asarray(sh["light_to_world"], np.float64).reshape(-1)[:12]
                arr[i].light_to_world = (ctypes.c_float * 12)(*lm.tolist())
                arr[i].flags |= _abi.SHAPE_LIGHT_TRANSFORM
        h.keep.append(arr)
        d.shapes = ctypes.cast(arr, ctypes.c_void_p)
        d.shape_count = len(shapes)
    if delta_lights:
        arr = (_abi.Light * len(delta_lights))()
        for i, li in enumerate(delta_lights):
            arr[i].kind = li["kind"]
            arr[i].rgb = (ctypes.c_float * 3)(*li["rgb"])
            arr[i].vec = (ctypes.c_float * 3)(*li["vec"])
        h.keep.append(arr)
        d.lights = ctypes.cast(arr, ctypes.c_void_p)
        d.light_count = len(delta_lights)
    return h


class Scene:
    """A scene resident on the current CUDA device (dort_gpu_scene_create)."""

    def __init__(self, verts, tris, **kw):
        self._holder = scene_desc(verts, tris, **kw)
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().dort_gpu_scene_create(ctypes.byref(self._holder.desc),
                                                    ctypes.byref(h)))
        self.handle = h
        self.tri_count = self._holder.desc.tri_count

    def close(self):
        if getattr(self, "handle", None) and _abi is not None:
            _abi.lib().dort_gpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def stats(self) -> dict:
        out = (ctypes.c_double * 8)()
        _abi.check(_abi.lib().dort_gpu_scene_stats(self.handle, out))
        return {"nodes": int(out[0]), "depth": int(out[1]), "tris": int(out[2]),
                "emissive": int(out[3]), "device_bytes": int(out[4]),
                "build_ms": out[5],
                "bvh_build": {_abi.BVH_BUILD_HOST: "host", _abi.BVH_BUILD_DEVICE: "device",
                              _abi.BVH_BUILD_PLOC: "ploc"}.get(int(out[6]), "none"),
                "bvh_ms": out[7]}

    def bvh_cost(self) -> dict:
        """Surface-area cost of the scene's BVH (dort_gpu_scene_bvh_cost)."""
        out = (ctypes.c_double * 4)()
        _abi.check(_abi.lib().dort_gpu_scene_bvh_cost(self.handle, out))
        return {"sah": out[0], "nodes": int(out[1]), "leaf_slots": int(out[2]),
                "depth": int(out[3])}

    def raycast(self, rays, any_hit: bool = False):
        """Host arrays in and out (dort_gpu_raycast)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.uint32)
        tb = None if any_hit else np.zeros((n, 3), np.float32)
        _abi.check(_abi.lib().dort_gpu_raycast(self.handle, _ptr(rays), n, int(any_hit),
                                               _ptr(prim), _ptr(tb)))
        return prim if any_hit else (prim, tb)

    def raycast_device(self, d_rays: int, n: int, d_prim: int, d_tb: int | None,
                       any_hit: bool = False, stream: int = 0):
        """Device pointers (ints) on a CUDA stream handle (int)."""
        _abi.check(_abi.lib().dort_gpu_raycast_device(
            self.handle, ctypes.c_void_p(d_rays), n, int(any_hit), ctypes.c_void_p(d_prim),
            ctypes.c_void_p(d_tb) if d_tb else None, ctypes.c_void_p(stream)))

    def render(self, params: _abi.RenderParams):
        """dort_gpu_render: returns (image [h, w, 3] float32, stats dict)."""
        out = np.zeros((params.height, params.width, 3), np.float32)
        st = (ctypes.c_double * 4)()
        _abi.check(_abi.lib().dort_gpu_render(self.handle, ctypes.byref(params), _ptr(out), st))
        return out, {"rays": st[0], "samples": st[1], "ms": st[2], "dropped": st[3]}

    def render_wavefront(self, params: _abi.RenderParams, tuning: dict | None = None):
        """dort_gpu_render_wavefront: returns (image, stats dict)."""
        out = np.zeros((params.height, params.width, 3), np.float32)
        st = (ctypes.c_double * 4)()
        t = wavefront_tuning(**tuning) if tuning else None
        _abi.check(_abi.lib().dort_gpu_render_wavefront(
            self.handle, ctypes.byref(params), ctypes.byref(t) if t else None, _ptr(out), st))
        return out, {"rays": st[0], "ms": st[2], "waves": st[3]}

    def render_wavefront_device(self, params: _abi.RenderParams, d_out: int, stream: int = 0,
                                tuning: dict | None = None):
        t = wavefront_tuning(**tuning) if tuning else None
        _abi.check(_abi.lib().dort_gpu_render_wavefront_device(
            self.handle, ctypes.byref(params), ctypes.byref(t) if t else None,
            ctypes.c_void_p(d_out), ctypes.c_void_p(stream)))

    def wavefront_stage_times(self, params: _abi.RenderParams, tuning: dict | None = None):
        """Per-stage milliseconds of one frame run wave by wave (measurement)."""
        ms = (ctypes.c_double * 6)()
        rays = (ctypes.c_double * 4)()
        t = wavefront_tuning(**tuning) if tuning else None
        _abi.check(_abi.lib().dort_gpu_wavefront_stage_times(
            self.handle, ctypes.byref(params), ctypes.byref(t) if t else None, ms, rays))
        names = ["regen", "extend", "shade", "shadow", "neeb"]
        out = {n: ms[i] for i, n in enumerate(names)}
        out["waves"] = ms[5]
        out["rays"] = rays[0]
        out["extend_rays"], out["shadow_rays"], out["neeb_rays"] = rays[1], rays[2], rays[3]
        return out

    def adjoint_forward(self, params: _abi.RenderParams, tri_albedo=None, tri_emission=None):
        """dort_gpu_adjoint_forward: image with per-triangle overrides."""
        out = np.zeros((params.height, params.width, 3), np.float32)
        a = None if tri_albedo is None else np.ascontiguousarray(tri_albedo, np.float32)
        e = None if tri_emission is None else np.ascontiguousarray(tri_emission, np.float32)
        _abi.check(_abi.lib().dort_gpu_adjoint_forward(self.handle, ctypes.byref(params),
                                                       _ptr(a), _ptr(e), _ptr(out)))
        return out

    def adjoint_backward(self, params: _abi.RenderParams, dl_dimage, tri_albedo=None,
                         tri_emission=None, want_albedo=True, want_emission=True):
        """dort_gpu_adjoint_backward: (d_albedo, d_emission), tri_count x 3 each."""
        g = np.ascontiguousarray(dl_dimage, np.float32)
        a = None if tri_albedo is None else np.ascontiguousarray(tri_albedo, np.float32)
        e = None if tri_emission is None else np.ascontiguousarray(tri_emission, np.float32)
        da = np.zeros((self.tri_count, 3), np.float32) if want_albedo else None
        de = np.zeros((self.tri_count, 3), np.float32) if want_emission else None
        _abi.check(_abi.lib().dort_gpu_adjoint_backward(self.handle, ctypes.byref(params),
                                                        _ptr(a), _ptr(e), _ptr(g), _ptr(da),
                                                        _ptr(de)))
        return da, de

    def adjoint_stats(self) -> dict:
        """dort_gpu_adjoint_stats: the last backward pass's engine ("wavefront",
        "megakernel" or "wavefront+megakernel"), samples traced a second time,
        wavefront rays and waves."""
        st = (ctypes.c_double * 4)()
        _abi.check(_abi.lib().dort_gpu_adjoint_stats(self.handle, st))
        return {"engine": ("wavefront", "megakernel", "wavefront+megakernel")[int(st[0])],
                "retraced": int(st[1]), "rays": st[2], "waves": int(st[3])}

    def render_device_noalloc(self, params: _abi.RenderParams, d_out: int, stream: int = 0):
        """dort_gpu_render_device_noalloc: no device allocation in the call."""
        _abi.check(_abi.lib().dort_gpu_render_device_noalloc(
            self.handle, ctypes.byref(params), ctypes.c_void_p(d_out), ctypes.c_void_p(stream)))

    def render_device(self, params: _abi.RenderParams, d_out: int, stream: int = 0):
        _abi.check(_abi.lib().dort_gpu_render_device(self.handle, ctypes.byref(params),
                                                     ctypes.c_void_p(d_out),
                                                     ctypes.c_void_p(stream)))

    def raycast_timed(self, d_rays: int, n: int, d_prim: int, d_tb: int | None,
                      any_hit: bool = False, stream: int = 0, repeat: int = 1) -> float:
        ms = ctypes.c_float(0.0)
        _abi.check(_abi.lib().dort_gpu_raycast_timed(
            self.handle, ctypes.c_void_p(d_rays), n, int(any_hit), ctypes.c_void_p(d_prim),
            ctypes.c_void_p(d_tb) if d_tb else None, ctypes.c_void_p(stream), repeat,
            ctypes.byref(ms)))
        return ms.value


def render_params(camera: dict, width: int, height: int, iterations: int = 1,
                  min_depth: int = 0, max_depth: int = 5, only_direct: bool = False,
                  sample_all_lights: bool = False, direct_strategy: str = "mis",
                  seed: int = 42, renderer: str = "pt",
                  use_t1_paths: bool = True, roulette: bool = True,
                  adjoint_megakernel: bool = False) -> _abi.RenderParams:
    """dort.render.make parameters (lua_render.cpp:102-160) with its defaults;
    `renderer` "pt" (the path tracer), "lt" / "light" (the light tracer) or
    "bdpt" (the bidirectional path tracer, with use_t1_paths).  roulette=False
    turns off the path tracer's Russian roulette (for derivative checks);
    adjoint_megakernel=True runs the adjoint's backward pass as a megakernel
    instead of the wavefront."""
    p = _abi.RenderParams()
    p.struct_size = ctypes.sizeof(_abi.RenderParams)
    p.width, p.height, p.iterations = width, height, iterations
    p.min_depth, p.max_depth = min_depth, max_depth
    p.only_direct, p.sample_all_lights = int(only_direct), int(sample_all_lights)
    p.direct_strategy = {"mis": 0, "bsdf": 1, "light": 2}[direct_strategy]
    p.seed = seed
    p.renderer = {"pt": _abi.RENDERER_PT, "path": _abi.RENDERER_PT, "lt": _abi.RENDERER_LT,
                  "light": _abi.RENDERER_LT, "bdpt": _abi.RENDERER_BDPT}[renderer]
    p.renderer_flags = ((0 if use_t1_paths else _abi.BDPT_NO_T1_PATHS) |
                        (0 if roulette else _abi.PT_NO_ROULETTE) |
                        (_abi.ADJOINT_MEGAKERNEL if adjoint_megakernel else 0))
    c = p.camera
    c.origin = (ctypes.c_float * 3)(*camera["origin"])
    c.right = (ctypes.c_float * 3)(*camera["right"])
    c.up = (ctypes.c_float * 3)(*camera["up"])
    c.forward = (ctypes.c_float * 3)(*camera["forward"])
    c.fov = camera.get("fov", 0.0)
    c.kind = camera.get("kind", _abi.CAMERA_PINHOLE)
    c.lens_radius = camera.get("lens_radius", 0.0)
    c.focal_distance = camera.get("focal_distance", 0.0)
    c.dimension = camera.get("dimension", 0.0)
    return p


def wavefront_tuning(queue_capacity: int = 0, trace_block: int = 0,
                     shade_block: int = 0, sort_rays: bool | None = None,
                     max_waves: int = 0,
                     stage_queues: bool | None = None,
                     deterministic: bool | None = None) -> _abi.WavefrontTuning:
    """dort_wavefront_tuning; zeros select the library's automatic choices.
    max_waves caps the waves of a frame (a frame that reaches it stops with
    DORT_ERR_TIMEOUT); stage_queues stages the shadow queue through bulk
    copies (TMA) into shared memory; deterministic adds the frame's per-unit
    sums in a fixed order (the same frame renders to the same bits)."""
    t = _abi.WavefrontTuning()
    t.struct_size = ctypes.sizeof(_abi.WavefrontTuning)
    t.queue_capacity, t.trace_block, t.shade_block = queue_capacity, trace_block, shade_block
    t.sort_rays = 0 if sort_rays is None else (1 if sort_rays else 2)
    t.max_waves = max_waves
    t.stage_queues = 0 if stage_queues is None else (1 if stage_queues else 2)
    t.deterministic = 0 if deterministic is None else (1 if deterministic else 2)
    return t


def bsdf_probe(material: dict, wo, wi=None, u=None, device: bool = True) -> dict:
    """dort_gpu_bsdf_probe: the BxDF code of one material (a dict as in
    scene_desc's materials) on local-frame directions.  Returns f and pdf of
    (wi, wo) when wi is given, and the sampled direction, its f and pdf when
    the uniforms u (n x 3) are given.  device=False runs the code compiled for
    the host."""
    m = _abi.Material()
    m.kind = material.get("kind", MAT_LAMBERT)
    m.color = (ctypes.c_float * 3)(*material.get("color", (0.0, 0.0, 0.0)))
    m.color2 = (ctypes.c_float * 3)(*material.get("color2", (0.0, 0.0, 0.0)))
    p = list(material.get("param", ())) + [0.0] * 4
    m.param = (ctypes.c_float * 4)(*p[:4])
    wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
    n = len(wo)
    out = {}
    if wi is not None:
        wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
        out["f"] = np.zeros((n, 3), np.float32)
        out["pdf"] = np.zeros(n, np.float32)
    if u is not None:
        u = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
        out["wi"] = np.zeros((n, 3), np.float32)
        out["sf"] = np.zeros((n, 3), np.float32)
        out["spdf"] = np.zeros(n, np.float32)
    _abi.check(_abi.lib().dort_gpu_bsdf_probe(
        ctypes.byref(m), n, _ptr(wo), _ptr(wi), _ptr(u), _ptr(out.get("f")),
        _ptr(out.get("pdf")), _ptr(out.get("wi")), _ptr(out.get("sf")),
        _ptr(out.get("spdf")), int(device)))
    return out


def debug_adjoint_list(entries: int) -> None:
    """dort_gpu_debug_adjoint_list: caps the backward pass's list of samples
    traced a second time (negative: the default); for tests."""
    _abi.check(_abi.lib().dort_gpu_debug_adjoint_list(int(entries)))


def debug_fail_alloc(after: int) -> None:
    """Failure injection (dort_gpu_debug_fail_alloc): the library's next
    `after` allocations succeed and the one after fails as if memory were
    exhausted; a negative value switches injection off."""
    _abi.check(_abi.lib().dort_gpu_debug_fail_alloc(int(after)))


def scene_from_dict(d: dict, **kw) -> "Scene":
    """Scene from the dict form used by dort_b200.scenes generators."""
    args = {k: d[k] for k in SCENE_KEYS if k in d and d[k] is not None}
    args.update(kw)
    return Scene(d["verts"], d["tris"], **args)


def host_check_render(d: dict, params: _abi.RenderParams, rows=None):
    """Runs the device path sampler compiled for the host (diagnostic)."""
    h = scene_desc(d["verts"], d["tris"],
                   **{k: d[k] for k in SCENE_KEYS if k in d and d[k] is not None})
    out = np.zeros((params.height, params.width, 3), np.float32)
    r0, r1 = rows if rows else (0, params.height)
    _abi.check(_abi.lib().dort_gpu_host_check_render(ctypes.byref(h.desc), ctypes.byref(params),
                                                     r0, r1, _ptr(out)))
    return out


class Batch:
    """Many frames rendered by one wavefront (dort_gpu_batch_*).  jobs is a
    list of (Scene, RenderParams); the scenes must outlive the batch."""

    def __init__(self, jobs, tuning: dict | None = None):
        arr = (_abi.BatchJob * len(jobs))()
        for i, (sc, p) in enumerate(jobs):
            arr[i].scene = sc.handle
            arr[i].params = p
        self._scenes = [sc for sc, _ in jobs]
        self._params = [p for _, p in jobs]
        t = wavefront_tuning(**tuning) if tuning else None
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().dort_gpu_batch_create(arr, len(jobs), ctypes.byref(t) if t else None,
                                                    ctypes.byref(h)))
        self.handle = h

    def render(self, stream: int = 0):
        _abi.check(_abi.lib().dort_gpu_batch_render(self.handle, ctypes.c_void_p(stream)))

    def image(self, job: int):
        p = self._params[job]
        out = np.zeros((p.height, p.width, 3), np.float32)
        _abi.check(_abi.lib().dort_gpu_batch_image(self.handle, job, _ptr(out)))
        return out

    def stats(self) -> dict:
        out = (ctypes.c_double * 4)()
        _abi.check(_abi.lib().dort_gpu_batch_stats(self.handle, out))
        return {"rays": out[0], "waves": out[1], "error": out[2], "samples": out[3]}

    def close(self):
        if getattr(self, "handle", None):
            _abi.lib().dort_gpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def loss_l2(image, target):
    """dort_gpu_loss_l2: (sum (image - target)^2, its image gradient)."""
    a = np.ascontiguousarray(image, np.float32)
    b = np.ascontiguousarray(target, np.float32)
    g = np.zeros_like(a)
    loss = ctypes.c_double(0.0)
    _abi.check(_abi.lib().dort_gpu_loss_l2(_ptr(a), _ptr(b), a.size, ctypes.byref(loss), _ptr(g)))
    return loss.value, g


def check_device_bvh(verts, tris, bvh_width: int = 8, bvh_build: str | None = None) -> dict:
    """Builds the BVH on the device ("device" = binned SAH, or "ploc") and
    compares it with the host collapse of the same binary tree
    (dort_gpu_check_device_bvh)."""
    h = scene_desc(verts, tris, bvh_width=bvh_width, bvh_build=bvh_build)
    out = (ctypes.c_double * 8)()
    _abi.check(_abi.lib().dort_gpu_check_device_bvh(ctypes.byref(h.desc), out))
    return {"node_bytes_differ": int(out[0]), "tri_bytes_differ": int(out[1]),
            "nodes": int(out[2]), "each_tri_once": bool(out[3]), "build_ms": out[4],
            "iterations": int(out[5]), "depth": int(out[6]), "sah": out[7]}


def host_check_raycast(verts, tris, rays, any_hit: bool = False, bvh_width: int = 8,
                       watertight: bool = False):
    """Runs the device traversal code compiled for the host (diagnostic)."""
    h = scene_desc(verts, tris, bvh_width=bvh_width, watertight=watertight)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = len(rays)
    prim = np.zeros(n, np.uint32)
    tb = None if any_hit else np.zeros((n, 3), np.float32)
    depth = ctypes.c_uint32(0)
    _abi.check(_abi.lib().dort_gpu_host_check_raycast(ctypes.byref(h.desc), _ptr(rays), n,
                                                      int(any_hit), _ptr(prim), _ptr(tb),
                                                      ctypes.byref(depth)))
    if any_hit:
        return prim, depth.value
    return prim, tb, depth.value
