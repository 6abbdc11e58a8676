"""ctypes bindings for the test oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, always as the checker or the timed CPU baseline,
never by the product package.

Two libraries:
  * ``liboracle.so`` -- the C restatement in oracle/*.c (always present once
    oracle/Makefile ran).
  * ``_ref/libdort_ref.so`` -- the reference renderer's own sources compiled
    with the harnesses in oracle/ref/ (present when the reference tree was
    available at build time; the built file travels with the repository).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdort_ref.so")

_P = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int


def build(ref_dir: str | None = None) -> None:
    """Compiles liboracle.so (and the reference harness when the reference
    tree exists)."""
    args = ["make", "-s", "-C", HERE]
    if ref_dir:
        args.append(f"REF={ref_dir}")
    subprocess.run(args, check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_bvh_build.restype = _P
        L.orc_bvh_build.argtypes = [_P, _u32, _P, _u32, _i32, _u32, _u32]
        L.orc_bvh_free.argtypes = [_P]
        L.orc_bvh_node_count.restype = _u32
        L.orc_bvh_node_count.argtypes = [_P]
        L.orc_bvh_nodes.argtypes = [_P, _P, _P]
        L.orc_raycast.argtypes = [_P, _P, _u64, _i32, _P, _P, _P, _P]
        L.orc_raycast_brute.argtypes = [_P, _P, _u32, _P, _u64, _P, _P]
        L.orc_triangle_hit.restype = _i32
        L.orc_triangle_hit.argtypes = [_P, _P, _P, _P, _P]
        L.orc_pt64.restype = _i32
        L.orc_pt64.argtypes = [_P, _u32, _P, _u32, _P, _P, _P, _P, ctypes.c_float, _u32, _u32,
                               _u32, _u32, _u32, _u64, _u32, _P, _P, _P, _P, _P]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_SO)
        R.dref_scene_create.restype = _P
        R.dref_scene_create.argtypes = [_P, _u32, _P, _u32, _i32, _u32, _u32, _u32, _P]
        R.dref_scene_destroy.argtypes = [_P]
        R.dref_raycast.restype = _i32
        R.dref_raycast.argtypes = [_P, _P, _u64, _i32, _u32, _P, _P, _P, _P]
        _ref = R
    return _ref


def _ggx_lib():
    R = ref()
    for name in ("dref_ggx_d", "dref_ggx_g1", "dref_ggx_sample_m"):
        getattr(R, name).restype = None
    R.dref_ggx_d.argtypes = [ctypes.c_float, ctypes.c_size_t, _P, _P]
    R.dref_ggx_g1.argtypes = [ctypes.c_float, ctypes.c_size_t, _P, _P, _P]
    R.dref_ggx_sample_m.argtypes = [ctypes.c_float, ctypes.c_size_t, _P, _P, _P]
    return R


def ref_ggx_d(alpha: float, m) -> np.ndarray:
    """The reference's MicrofacetDistrib(GGX, alpha).d(m) in float
    (microfacet.cpp:19-36)."""
    m = np.ascontiguousarray(m, np.float32).reshape(-1, 3)
    out = np.zeros(len(m), np.float32)
    _ggx_lib().dref_ggx_d(alpha, len(m), _ptr(m), _ptr(out))
    return out


def ref_ggx_g1(alpha: float, v, m) -> np.ndarray:
    """The reference's MicrofacetDistrib(GGX, alpha).g1(v, m)
    (microfacet.cpp:38-58)."""
    v = np.ascontiguousarray(v, np.float32).reshape(-1, 3)
    m = np.ascontiguousarray(m, np.float32).reshape(-1, 3)
    out = np.zeros(len(v), np.float32)
    _ggx_lib().dref_ggx_g1(alpha, len(v), _ptr(v), _ptr(m), _ptr(out))
    return out


def ref_ggx_sample_m(alpha: float, uv) -> tuple[np.ndarray, np.ndarray]:
    """The reference's MicrofacetDistrib(GGX, alpha).sample_m(uv, pdf)
    (microfacet.cpp:64-86): half vectors and pdfs."""
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    m = np.zeros((len(uv), 3), np.float32)
    pdf = np.zeros(len(uv), np.float32)
    _ggx_lib().dref_ggx_sample_m(alpha, len(uv), _ptr(uv), _ptr(m), _ptr(pdf))
    return m, pdf


def _mesh_args(verts, tris):
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
    tris = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
    return verts, tris


class OracleBvh:
    """The C restatement of the reference's binary BVH (bvh.cpp:9-469)."""

    def __init__(self, verts, tris, split: str = "sah", leaf_size: int = 6,
                 max_leaf_size: int = 32):
        self.verts, self.tris = _mesh_args(verts, tris)
        m = {"middle": 0, "sah": 1}[split]
        self.h = lib().orc_bvh_build(_ptr(self.verts), len(self.verts),
                                     _ptr(self.tris), len(self.tris), m,
                                     leaf_size, max_leaf_size)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_free(self.h)
            self.h = None

    def node_count(self) -> int:
        return lib().orc_bvh_node_count(self.h)

    def nodes(self):
        n = self.node_count()
        boxes = np.zeros((n, 6), np.float32)
        meta = np.zeros((n, 3), np.uint32)
        lib().orc_bvh_nodes(self.h, _ptr(boxes), _ptr(meta))
        return boxes, meta

    def raycast(self, rays, any_hit: bool = False, counts: bool = False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.uint32)
        tb = np.zeros((n, 3), np.float32)
        nodes = np.zeros(n, np.uint32) if counts else None
        tests = np.zeros(n, np.uint32) if counts else None
        lib().orc_raycast(self.h, _ptr(rays), n, int(any_hit), _ptr(prim),
                          _ptr(tb), _ptr(nodes), _ptr(tests))
        if counts:
            return prim, tb, nodes, tests
        return prim, tb


def brute_raycast(verts, tris, rays):
    verts, tris = _mesh_args(verts, tris)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    prim = np.zeros(len(rays), np.uint32)
    tb = np.zeros((len(rays), 3), np.float32)
    lib().orc_raycast_brute(_ptr(verts), _ptr(tris), len(tris), _ptr(rays),
                            len(rays), _ptr(prim), _ptr(tb))
    return prim, tb


def triangle_hit(p0, p1, p2, ray):
    a = [np.ascontiguousarray(x, dtype=np.float32) for x in (p0, p1, p2, ray)]
    tb = np.zeros(3, np.float32)
    ok = lib().orc_triangle_hit(*[_ptr(x) for x in a], _ptr(tb))
    return bool(ok), tb


def pt64(scene: dict, width: int, height: int, spp: int, max_depth: int, seed: int,
         albedo, emission, dl_dimage=None, min_depth: int = 0, no_roulette: bool = False):
    """The float64 restatement of the "pt" estimator (oracle/pt64.c) on a
    Lambert triangle scene with triangle emitters (the adjoint workload's
    kind): the image, and with dl_dimage the loss gradients with respect to
    per-triangle albedo and emission.  `scene` carries verts, tris, camera and
    tri_emission (the emission it was created with); albedo / emission are
    the per-triangle values in effect."""
    v, t = _mesh_args(scene["verts"], scene["tris"])
    alb = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
    em = np.ascontiguousarray(emission, np.float32).reshape(-1, 3)
    em0 = np.ascontiguousarray(scene["tri_emission"], np.float32).reshape(-1, 3)
    cam = pack_camera(scene["camera"])
    img = np.zeros((height, width, 3), np.float64)
    g = None if dl_dimage is None else np.ascontiguousarray(dl_dimage, np.float32)
    da = np.zeros((len(t), 3), np.float64) if g is not None else None
    de = np.zeros((len(t), 3), np.float64) if g is not None else None
    rays = ctypes.c_uint64(0)
    rc = lib().orc_pt64(_ptr(v), len(v), _ptr(t), len(t), _ptr(alb), _ptr(em), _ptr(em0),
                        _ptr(cam), ctypes.c_float(scene["camera"]["fov"]), width, height, spp,
                        min_depth, max_depth, seed, int(no_roulette), _ptr(g), _ptr(img),
                        _ptr(da), _ptr(de), ctypes.byref(rays))
    if rc != 0:
        raise ValueError("orc_pt64: bad triangle index")
    return img, da, de


class RefBvh:
    """The reference's own Bvh<> + Triangle code (compiled from its sources)."""

    def __init__(self, verts, tris, split: str = "sah", leaf_size: int = 6,
                 max_leaf_size: int = 32, threads: int = 1):
        self.verts, self.tris = _mesh_args(verts, tris)
        m = {"middle": 0, "sah": 1}[split]
        bt = ctypes.c_double(0.0)
        self.h = ref().dref_scene_create(_ptr(self.verts), len(self.verts),
                                         _ptr(self.tris), len(self.tris), m,
                                         leaf_size, max_leaf_size, threads,
                                         ctypes.byref(bt))
        self.build_s = bt.value

    def __del__(self):
        if getattr(self, "h", None):
            ref().dref_scene_destroy(self.h)
            self.h = None

    def raycast(self, rays, any_hit: bool = False, threads: int = 1,
                counts: bool = False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        prim = np.zeros(n, np.uint32)
        tb = np.zeros((n, 3), np.float32)
        tests = np.zeros(n, np.uint32) if counts else None
        ts = ctypes.c_double(0.0)
        ref().dref_raycast(self.h, _ptr(rays), n, int(any_hit), threads,
                           _ptr(prim), _ptr(tb), _ptr(tests), ctypes.byref(ts))
        self.trace_s = ts.value
        if counts:
            return prim, tb, tests
        return prim, tb


def pack_materials(materials) -> np.ndarray:
    """Material dicts -> rows of 11 floats (kind, color[3], color2[3], param[4])."""
    rows = []
    for m in materials:
        p = list(m.get("param", ())) + [0.0] * 4
        rows.append([float(m.get("kind", 0)), *m.get("color", (0, 0, 0)),
                     *m.get("color2", (0, 0, 0)), *p[:4]])
    return np.ascontiguousarray(np.array(rows, np.float32).reshape(-1, 11))


def pack_camera(cam) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate(
        [cam["origin"], cam["right"], cam["up"], cam["forward"]]).astype(np.float32))


def ref_pt_render(scene: dict, width: int, height: int, iterations: int,
                  min_depth: int = 0, max_depth: int = 5, only_direct: bool = False,
                  sample_all_lights: bool = False, strategy: str = "mis", seed: int = 42,
                  split: str = "middle", threads: int | None = None):
    """Renders with the reference's own PathRenderer (dort.render.make with
    renderer = "pt"); returns (image [h, w, 3] f32, seconds)."""
    R = ref()
    if not hasattr(R, "_pt_ready"):
        R.dref_pt_render.restype = _i32
        R.dref_pt_render.argtypes = [_P, _u32, _P, _u32, _P, _P, _u32, _P, _P, _P, _u32,
                                     _u32, _P, _P, ctypes.c_float, _u32, _u32, _u32, _u32,
                                     _u32, _i32, _i32, _i32, _u32, _i32, _u32, _P, _P]
        R._pt_ready = True
    v = np.ascontiguousarray(scene["verts"], np.float32)
    t = np.ascontiguousarray(scene["tris"], np.uint32)
    tm = np.ascontiguousarray(scene.get("tri_material", np.zeros(len(t), np.uint32)), np.uint32)
    mats = pack_materials(scene["materials"])
    em = scene.get("tri_emission")
    em = None if em is None else np.ascontiguousarray(em, np.float32)
    bg = scene.get("sky_const")
    bg = None if bg is None else np.ascontiguousarray(bg, np.float32)
    env = scene.get("sky_rgb")
    env_frame = None
    ew = eh = 0
    if env is not None:
        env = np.ascontiguousarray(env, np.float32)
        eh, ew = env.shape[0], env.shape[1]
        env_frame = np.ascontiguousarray(np.concatenate([
            np.asarray(scene.get("sky_scale", (1, 1, 1)), np.float32),
            np.asarray(scene.get("sky_up", (0, 1, 0)), np.float32),
            np.asarray(scene.get("sky_fwd", (1, 0, 0)), np.float32)]))
    cam = pack_camera(scene["camera"])
    out = np.zeros((height, width, 3), np.float32)
    secs = ctypes.c_double(0.0)
    strat = {"mis": 0, "bsdf": 1, "light": 2}[strategy]
    R.dref_pt_render(_ptr(v), len(v), _ptr(t), len(t), _ptr(tm), _ptr(mats), len(mats),
                     _ptr(em), _ptr(bg), _ptr(env), ew, eh, _ptr(env_frame), _ptr(cam),
                     ctypes.c_float(scene["camera"]["fov"]), width, height, iterations,
                     min_depth, max_depth, int(only_direct), int(sample_all_lights), strat,
                     seed, {"middle": 0, "sah": 1}[split], threads or os.cpu_count() or 1,
                     _ptr(out), ctypes.byref(secs))
    return out, secs.value


class RefPtScene:
    """A scene built once by the reference (for repeated timed renders)."""

    def __init__(self, scene: dict, split: str = "middle", threads: int = 1):
        R = ref()
        if not hasattr(R, "_pts_ready"):
            R.dref_pt_scene_create.restype = _P
            R.dref_pt_scene_create.argtypes = [_P, _u32, _P, _u32, _P, _P, _u32, _P, _P, _P,
                                               _u32, _u32, _P, _i32, _u32, _P]
            R.dref_pt_scene_destroy.argtypes = [_P]
            R.dref_pt_scene_render.restype = _i32
            R.dref_pt_scene_render.argtypes = [_P, _P, ctypes.c_float, _u32, _u32, _u32, _u32,
                                               _u32, _i32, _i32, _i32, _u32, _u32, _P, _P]
            R._pts_ready = True
        self.keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            self.keep.append(a)
            return a
        v = arr(scene["verts"], np.float32)
        t = arr(scene["tris"], np.uint32)
        tm = arr(scene.get("tri_material"), np.uint32)
        mats = arr(pack_materials(scene["materials"]), np.float32)
        em = arr(scene.get("tri_emission"), np.float32)
        bg = arr(scene.get("sky_const"), np.float32)
        env = arr(scene.get("sky_rgb"), np.float32)
        ew = eh = 0
        frame = None
        if env is not None:
            eh, ew = env.shape[0], env.shape[1]
            frame = arr(np.concatenate([
                np.asarray(scene.get("sky_scale", (1, 1, 1)), np.float32),
                np.asarray(scene.get("sky_up", (0, 1, 0)), np.float32),
                np.asarray(scene.get("sky_fwd", (1, 0, 0)), np.float32)]), np.float32)
        bs = ctypes.c_double(0.0)
        self.h = R.dref_pt_scene_create(_ptr(v), len(v), _ptr(t), len(t), _ptr(tm), _ptr(mats),
                                        len(mats), _ptr(em), _ptr(bg), _ptr(env), ew, eh,
                                        _ptr(frame), {"middle": 0, "sah": 1}[split], threads,
                                        ctypes.byref(bs))
        self.build_s = bs.value
        self.camera = scene["camera"]

    def render(self, width, height, iterations, min_depth=0, max_depth=5, seed=42,
               strategy="mis", threads=1):
        cam = pack_camera(self.camera)
        out = np.zeros((height, width, 3), np.float32)
        secs = ctypes.c_double(0.0)
        ref().dref_pt_scene_render(self.h, _ptr(cam), ctypes.c_float(self.camera["fov"]), width,
                                   height, iterations, min_depth, max_depth, 0, 0,
                                   {"mis": 0, "bsdf": 1, "light": 2}[strategy], seed, threads,
                                   _ptr(out), ctypes.byref(secs))
        return out, secs.value

    def __del__(self):
        if getattr(self, "h", None):
            ref().dref_pt_scene_destroy(self.h)
            self.h = None


def ref_scene_render(scene: dict, params) -> tuple[np.ndarray, float]:
    """Renders a scene dict (the form dort_b200.scene_desc takes: triangles,
    analytic shapes, delta lights, sky) with the reference's own PathRenderer
    (LightRenderer / BdptRenderer for params.renderer = lt / bdpt),
    single-threaded; `params` is a dort_b200 RenderParams (camera kind
    included).  Returns (image [h, w, 3] f32, seconds).  The ctypes structures
    of the product's C ABI only describe the input here; nothing of the
    product library runs."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from dort_b200 import SCENE_KEYS, scene_desc
    R = ref()
    if not hasattr(R, "_scene_ready"):
        R.dref_scene_render.restype = _i32
        R.dref_scene_render.argtypes = [_P, _P, _P, _P]
        R._scene_ready = True
    h = scene_desc(scene["verts"], scene["tris"],
                   **{k: scene[k] for k in SCENE_KEYS if k in scene and scene[k] is not None})
    out = np.zeros((params.height, params.width, 3), np.float32)
    secs = ctypes.c_double(0.0)
    R.dref_scene_render(ctypes.byref(h.desc), ctypes.byref(params), _ptr(out),
                        ctypes.byref(secs))
    return out, secs.value


def ref_read_ply(path: str) -> tuple[np.ndarray, np.ndarray]:
    """Reads a PLY file with the reference's read_ply_to_mesh (over the rply
    library it vendors).  Returns (points float32 (n, 3), vertex indices
    uint32 (3m,)); raises OSError / ValueError as the reference's callers
    fail."""
    R = ref()
    if not hasattr(R, "_ply_ready"):
        R.dref_read_ply.restype = _i32
        R.dref_read_ply.argtypes = [ctypes.c_char_p, _P, _u32, _P, _u32, _P]
        R._ply_ready = True
    counts = np.zeros(2, np.uint32)
    rc = R.dref_read_ply(path.encode(), None, 0, None, 0, _ptr(counts))
    if rc == -1:
        raise OSError(f"Could not open ply mesh file for reading: {path}")
    if rc != 0:
        raise ValueError(f"Could not read ply file: {path}")
    pts = np.zeros((int(counts[0]), 3), np.float32)
    verts = np.zeros(int(counts[1]), np.uint32)
    R.dref_read_ply(path.encode(), _ptr(pts), len(pts), _ptr(verts), len(verts), _ptr(counts))
    return pts, verts
