"""Scene builder: the reference's scene-description API over the flat scene.

Mirrors dort.builder and dort/dsl (src/dort/lua_builder.cpp,
lua/dort/dsl.lua, lua/dort/builder_ext.lua) and the constructors behind them
(dort.geometry, dort.shape, dort.material, dort.light, dort.camera:
lua_geometry.cpp, lua_shape.cpp, lua_material.cpp, lua_light.cpp,
lua_camera.cpp), with the reference's parameter names and defaults, and
records the scene the way the reference's primitive tree would hold it:

  - add_triangle(mesh, i)         TriangleShapePrimitive: mesh coordinates
                                  used directly (lua_builder.cpp:368-391)
  - add_shape(shape[, light])     ShapePrimitive with the current transform
                                  (lua_builder.cpp:316-348); a triangle
                                  shape's vertices are baked through it
  - frame / add_primitive         FramePrimitive instancing
                                  (lua_builder.cpp:177-220, 350-366),
                                  flattened by composing the transforms
  - mesh{points, vertices}        points taken through `transform` (default:
                                  the builder's, dsl.lua:150-155)
  - Builder.diffuse_light / point_light / directional_light /
    environment_light put the builder's transform in front of theirs, as the
    dsl's functions do (dsl.lua:109-136); the module-level constructors take
    the transform as given, as dort.light.make_* do
  - set_transform composes (local_to_frame = local_to_frame * t,
    lua_builder.cpp:227-232), which add_diffuse_light relies on: its shape
    ends up under builder * light transform while the light keeps its own
    (builder_ext.lua:38-48); the flat scene keeps both

build_scene() returns the flat scene dict the Scene constructor takes
(verts, tris, tri_material, materials, tri_emission, shapes, delta_lights,
sky_*)
and the default camera as a camera dict.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi, ply

# ---- geometry (transform.cpp:49-165; 4x4 matrices, column vectors) ---------


class Transform:
    __slots__ = ("m",)

    def __init__(self, m):
        self.m = np.asarray(m, np.float64).reshape(4, 4)

    def __mul__(self, other: "Transform") -> "Transform":
        return Transform(self.m @ other.m)

    def apply_point(self, p):
        p = np.asarray(p, np.float64)
        return self.m[:3, :3] @ p + self.m[:3, 3]

    def apply_points(self, p):
        """apply_point over the rows of an (n, 3) array."""
        return np.asarray(p, np.float64).reshape(-1, 3) @ self.m[:3, :3].T + self.m[:3, 3]

    def apply_vector(self, v):
        return self.m[:3, :3] @ np.asarray(v, np.float64)

    def inverse(self) -> "Transform":
        return Transform(np.linalg.inv(self.m))

    def rows3x4(self):
        return self.m[:3, :].reshape(-1)


def identity() -> Transform:
    return Transform(np.eye(4))


def translate(x, y=None, z=None) -> Transform:
    if y is None:
        x, y, z = x
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return Transform(m)


def scale(x, y=None, z=None) -> Transform:
    if y is None:
        y = z = x
    return Transform(np.diag([x, y, z, 1.0]))


def _rot(axis: int, angle: float) -> Transform:
    c, s = math.cos(angle), math.sin(angle)
    m = np.eye(4)
    i, j = [(1, 2), (2, 0), (0, 1)][axis]
    m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
    return Transform(m)


def rotate_x(angle: float) -> Transform:
    return _rot(0, angle)


def rotate_y(angle: float) -> Transform:
    return _rot(1, angle)


def rotate_z(angle: float) -> Transform:
    return _rot(2, angle)


def look_at(eye, look, up) -> Transform:
    """Camera-to-world (or object-to-world) frame at `eye` looking at `look`
    (transform.cpp:146-165): columns right = normalize(up x dir), up' = dir x
    right, dir."""
    eye, look, up = (np.asarray(a, np.float64) for a in (eye, look, up))
    d = look - eye
    d = d / np.linalg.norm(d)
    r = np.cross(up / np.linalg.norm(up), d)
    r = r / np.linalg.norm(r)
    u = np.cross(d, r)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = r, u, d, eye
    return Transform(m)


def point(x, y, z):
    return np.array([x, y, z], np.float64)


vector = point


def rgb(r, g=None, b=None):
    """dort.spectrum.rgb: rgb(x) or rgb(r, g, b)."""
    if g is None:
        return np.array([r, r, r], np.float64)
    return np.array([r, g, b], np.float64)


def rgbh(hexval):
    """dort.spectrum.rgbh(0xRRGGBB) (lua_spectrum.cpp:62-101)."""
    if isinstance(hexval, str):
        hexval = int(hexval.lstrip("#"), 16)
    return np.array([(hexval >> 16) & 0xFF, (hexval >> 8) & 0xFF, hexval & 0xFF],
                    np.float64) / 255.0


# ---- materials (lua_material.cpp; defaults as there) ------------------------


class Material:
    __slots__ = ("kind", "color", "color2", "param")

    def __init__(self, kind, color=(0, 0, 0), color2=(0, 0, 0), param=()):
        self.kind = kind
        self.color = tuple(float(c) for c in color)
        self.color2 = tuple(float(c) for c in color2)
        self.param = tuple(float(p) for p in param)

    def key(self):
        return (self.kind, self.color, self.color2, self.param)

    def as_dict(self):
        return {"kind": self.kind, "color": self.color, "color2": self.color2,
                "param": self.param}


def lambert_material(albedo=rgb(1.0)):
    return Material(_abi.MAT_LAMBERT, albedo)


def oren_nayar_material(albedo=rgb(1.0), sigma=0.1):
    return Material(_abi.MAT_OREN_NAYAR, albedo, param=(sigma,))


def mirror_material(albedo=rgb(1.0)):
    return Material(_abi.MAT_MIRROR, albedo)


def dielectric_material(reflect_tint=rgb(1.0), transmit_tint=rgb(1.0), ior_inside=1.5,
                        ior_outside=1.0, is_thin=False):
    return Material(_abi.MAT_DIELECTRIC, reflect_tint, transmit_tint,
                    (ior_inside, ior_outside, 1.0 if is_thin else 0.0))


def phong_material(albedo=rgb(0.0), glossy_albedo=None, exponent=50.0):
    glossy = albedo if glossy_albedo is None else glossy_albedo
    return Material(_abi.MAT_PHONG, albedo, glossy, (exponent,))


def conductor_material(f0=rgb(1.0), alpha=0.1):
    """GGX conductor (no reference counterpart)."""
    return Material(_abi.MAT_CONDUCTOR, f0, param=(alpha,))


# ---- shapes (lua_shape.cpp) -------------------------------------------------


class Mesh:
    __slots__ = ("points", "vertices")

    def __init__(self, points, vertices):
        self.points = np.asarray(points, np.float64).reshape(-1, 3)
        self.vertices = np.asarray(vertices, np.int64).reshape(-1)


class Shape:
    __slots__ = ("kind", "param", "mesh", "index")

    def __init__(self, kind, param=(), mesh=None, index=0):
        self.kind, self.param, self.mesh, self.index = kind, tuple(param), mesh, index


def read_ply_mesh(file_name) -> Mesh:
    """dort.shape.read_ply_mesh (lua_shape.cpp:225-241): the file's points
    (untransformed) and its faces fanned into triangles."""
    pts, verts = ply.read_ply(file_name)
    return Mesh(pts, verts)


def sphere(radius):
    return Shape(_abi.SHAPE_SPHERE, (radius,))


def disk(radius, z=0.0):
    return Shape(_abi.SHAPE_DISK, (radius, z))


def cube():
    return Shape(_abi.SHAPE_CUBE)


def cylinder(radius, z_min=-1.0, z_max=1.0):
    return Shape(_abi.SHAPE_CYLINDER, (radius, z_min, z_max))


# ---- lights (lua_light.cpp) --------------------------------------------------


class Light:
    __slots__ = ("kind", "data")

    def __init__(self, kind, **data):
        self.kind, self.data = kind, data


def point_light(point, intensity, transform=None):
    t = transform or identity()
    return Light("point", point=t.apply_point(point), intensity=np.asarray(intensity))


def directional_light(direction, radiance, transform=None):
    t = transform or identity()
    return Light("directional", direction=t.apply_vector(direction),
                 radiance=np.asarray(radiance))


def diffuse_light(shape, radiance, transform=None):
    return Light("diffuse", shape=shape, radiance=np.asarray(radiance),
                 transform=transform or identity())


def infinite_light(radiance):
    return Light("infinite", radiance=np.asarray(radiance))


def environment_light(image, up=(0, 1, 0), forward=(1, 0, 0), scale=rgb(1.0), transform=None):
    t = transform or identity()
    return Light("environment", image=np.asarray(image, np.float32),
                 up=t.apply_vector(up), forward=t.apply_vector(forward),
                 scale=np.asarray(scale))


# ---- cameras (lua_camera.cpp) -----------------------------------------------


def _camera(transform: Transform, **kw):
    m = transform.m
    return {"origin": tuple(m[:3, 3]), "right": tuple(m[:3, 0]), "up": tuple(m[:3, 1]),
            "forward": tuple(m[:3, 2]), **kw}


def pinhole_camera(transform, fov=math.pi * 0.5):
    return _camera(transform, fov=fov, kind=_abi.CAMERA_PINHOLE)


def ortho_camera(dimension, transform=None):
    return _camera(transform or identity(), dimension=dimension, kind=_abi.CAMERA_ORTHO)


def thin_lens_camera(transform, lens_radius, focal_distance, fov=math.pi * 0.5):
    return _camera(transform, fov=fov, lens_radius=lens_radius, focal_distance=focal_distance,
                   kind=_abi.CAMERA_THIN_LENS)


# ---- the builder (lua_builder.cpp) ------------------------------------------


class _Prim:
    __slots__ = ("kind", "shape", "material", "light", "transform", "frame")

    def __init__(self, kind, shape=None, material=None, light=None, transform=None, frame=None):
        self.kind, self.shape, self.material = kind, shape, material
        self.light, self.transform, self.frame = light, transform, frame


class Builder:
    """dort.builder state: current transform and material, the open frame,
    state and frame stacks, lights and the default camera."""

    def __init__(self):
        self.transform = identity()
        self.material = None
        self.frame = []
        self.state_stack = []
        self.frame_stack = []
        self.lights = []
        self.camera = None

    # state (lua_builder.cpp:149-270)
    def push_state(self):
        self.state_stack.append((self.transform, self.material))

    def pop_state(self):
        if not self.state_stack:
            raise ValueError("State stack is empty (not balanced)")
        self.transform, self.material = self.state_stack.pop()

    def block(self, callback):
        self.push_state()
        try:
            return callback()
        finally:
            self.pop_state()

    def set_transform(self, t: Transform):
        # replaces by composing: local_to_frame = local_to_frame * t
        self.transform = self.transform * t

    def get_transform(self) -> Transform:
        return self.transform

    def set_material(self, m: Material):
        self.material = m

    def set_camera(self, c: dict):
        self.camera = c

    # frames (lua_builder.cpp:177-220)
    def push_frame(self):
        self.state_stack.append((self.transform, self.material))
        self.frame_stack.append(self.frame)
        self.transform = identity()
        self.frame = []

    def pop_frame(self):
        if not self.frame_stack:
            raise ValueError("Frame stack is empty (not balanced)")
        prim = _Prim("frame", frame=self.frame)
        self.frame = self.frame_stack.pop()
        self.transform, self.material = self.state_stack.pop()
        return prim

    def frame_(self, callback):
        self.push_frame()
        callback()
        return self.pop_frame()

    # adding (lua_builder.cpp:316-415)
    def _need_material(self):
        if self.material is None:
            raise ValueError("no material is set")

    def add_shape(self, shape: Shape, light: Light | None = None):
        self._need_material()
        if light is not None and light.kind != "diffuse":
            raise ValueError("the light must be an area light")
        self.frame.append(_Prim("shape", shape=shape, material=self.material, light=light,
                                transform=self.transform))

    def add_triangle(self, mesh: Mesh, index: int):
        self._need_material()
        self.frame.append(_Prim("triangle", shape=Shape("tri", mesh=mesh, index=index),
                                material=self.material))

    def add_read_ply_mesh(self, file_name):
        """lua_builder.cpp:418-448: every triangle of the file as a separate
        primitive with the current material, its points taken through the
        builder's transform."""
        mesh = read_ply_mesh(file_name)
        self._need_material()
        self._add_mesh(mesh)

    def add_ply_mesh(self, mesh: Mesh):
        """lua_builder.cpp:501-525: the triangles of a mesh read by
        read_ply_mesh, its points taken through the builder's transform."""
        self._need_material()
        self._add_mesh(mesh)

    # one BVH per mesh in the reference (MeshBvhPrimitive); the same
    # triangles in the scene's one BVH here
    add_read_ply_mesh_as_bvh = add_read_ply_mesh
    add_ply_mesh_as_bvh = add_ply_mesh

    def _add_mesh(self, mesh: Mesh):
        pts = self.transform.apply_points(mesh.points)
        self.frame.append(_Prim("mesh", shape=Shape("tri", mesh=Mesh(pts, mesh.vertices)),
                                material=self.material))

    def add_primitive(self, prim: _Prim):
        self.frame.append(_Prim("instance", frame=prim.frame, transform=self.transform))

    def add_light(self, light: Light):
        if self.frame_stack:
            raise ValueError("lights can only be added in the root frame")
        self.lights.append(light)

    def add_diffuse_light(self, shape, radiance, transform=None):
        """dsl.add_diffuse_light + builder_ext.lua:38-48: the light (under
        the builder's transform times `transform`), and its shape with a
        black Lambert material, added after set_transform of that transform."""
        t = self._dsl_transform(transform)
        light = diffuse_light(shape, radiance, t)

        def body():
            self.set_transform(t)
            self.material = lambert_material(rgb(0.0))
            self.add_shape(shape, light)
        self.block(body)
        self.add_light(light)
        return light

    # dsl.lua:100-155: constructors that apply the builder's transform
    def _dsl_transform(self, transform):
        return self.transform * transform if transform is not None else self.transform

    def point_light(self, point, intensity, transform=None):
        return point_light(point, intensity, self._dsl_transform(transform))

    def directional_light(self, direction, radiance, transform=None):
        return directional_light(direction, radiance, self._dsl_transform(transform))

    def diffuse_light(self, shape, radiance, transform=None):
        return diffuse_light(shape, radiance, self._dsl_transform(transform))

    def environment_light(self, image, up=(0, 1, 0), forward=(1, 0, 0), scale=rgb(1.0),
                          transform=None):
        return environment_light(image, up, forward, scale, self._dsl_transform(transform))

    def mesh(self, points, vertices, transform=None):
        t = transform if transform is not None else self.transform
        return Mesh([t.apply_point(p) for p in np.asarray(points, np.float64).reshape(-1, 3)],
                    vertices)

    def triangle(self, mesh: Mesh, index: int) -> Shape:
        """dort.builder.make_triangle (lua_builder.cpp:655-667)."""
        return Shape("tri", mesh=mesh, index=index)

    # ---- flattening (build_scene, lua_builder.cpp:113-146) ----
    def build_scene(self) -> dict:
        if self.frame_stack:
            raise ValueError("Frame stack is not empty")
        if self.state_stack:
            raise ValueError("State stack is not empty")
        verts, tris, tri_mat, tri_em, light_verts = [], [], [], [], []
        shapes = []
        mats, mat_index = [], {}

        def mat_id(m: Material) -> int:
            k = m.key()
            if k not in mat_index:
                mat_index[k] = len(mats)
                mats.append(m.as_dict())
            return mat_index[k]

        lit_prims = set()
        any_light_verts = [False]

        def emit(prims, outer: Transform):
            for p in prims:
                if p.kind == "instance":
                    emit(p.frame, outer * p.transform)
                    continue
                if p.kind == "mesh":
                    # all triangles of a mesh at once, in index order
                    tri_vertices = p.shape.mesh.vertices[:len(p.shape.mesh.vertices) // 3 * 3]
                    n = len(tri_vertices) // 3
                    base = len(verts)
                    world = outer.apply_points(p.shape.mesh.points)[tri_vertices].tolist()
                    verts.extend(world)
                    light_verts.extend(world)
                    tris.extend((base + np.arange(3 * n)).reshape(-1, 3).tolist())
                    tri_mat.extend([mat_id(p.material)] * n)
                    tri_em.extend([(0.0, 0.0, 0.0)] * n)
                    continue
                em = (0.0, 0.0, 0.0)
                light_t = None
                if p.light is not None:
                    em = tuple(float(c) for c in p.light.data["radiance"])
                    lit_prims.add(id(p.light))
                    prim_t = outer * p.transform
                    if not np.allclose(p.light.data["transform"].m, prim_t.m, rtol=0, atol=0):
                        light_t = p.light.data["transform"]
                if p.kind == "triangle" or p.shape.kind == "tri":
                    mesh, i = p.shape.mesh, p.shape.index
                    t = outer if p.kind == "triangle" else outer * p.transform
                    base = len(verts)
                    for k in range(3):
                        src = mesh.points[mesh.vertices[i + k]]
                        verts.append(t.apply_point(src))
                        # the triangle the light samples (its own transform)
                        light_verts.append(verts[-1] if light_t is None
                                           else light_t.apply_point(src))
                    if light_t is not None:
                        any_light_verts[0] = True
                    tris.append((base, base + 1, base + 2))
                    tri_mat.append(mat_id(p.material))
                    tri_em.append(em)
                else:
                    t = outer * p.transform
                    shapes.append({"kind": p.shape.kind, "material": mat_id(p.material),
                                   "param": p.shape.param, "to_world": t.rows3x4(),
                                   "emission": em,
                                   "light_to_world": None if light_t is None
                                   else light_t.rows3x4()})

        emit(self.frame, identity())
        d = {"verts": np.asarray(verts, np.float32).reshape(-1, 3),
             "tris": np.asarray(tris, np.uint32).reshape(-1, 3),
             "tri_material": np.asarray(tri_mat, np.uint32),
             "materials": mats or [lambert_material(rgb(0.5)).as_dict()],
             "tri_emission": np.asarray(tri_em, np.float32).reshape(-1, 3),
             "shapes": shapes, "delta_lights": []}
        if any_light_verts[0]:
            d["tri_light_verts"] = np.asarray(light_verts, np.float32).reshape(-1, 9)
        sky = np.zeros(3)
        for light in self.lights:
            if light.kind == "point":
                d["delta_lights"].append({"kind": _abi.LIGHT_POINT, "rgb": light.data["intensity"],
                                    "vec": light.data["point"]})
            elif light.kind == "directional":
                d["delta_lights"].append({"kind": _abi.LIGHT_DIRECTIONAL,
                                    "rgb": light.data["radiance"],
                                    "vec": light.data["direction"]})
            elif light.kind == "infinite":
                sky = sky + light.data["radiance"]
            elif light.kind == "environment":
                if "sky_rgb" in d:
                    raise ValueError("at most one environment light")
                d["sky_rgb"] = light.data["image"]
                d["sky_scale"] = tuple(light.data["scale"])
                d["sky_up"] = tuple(light.data["up"])
                d["sky_fwd"] = tuple(light.data["forward"])
            elif light.kind == "diffuse":
                if id(light) not in lit_prims:
                    raise ValueError("a diffuse light must be added with its shape "
                                     "(add_shape(shape, light)); lights without geometry "
                                     "are not supported")
        d["sky_const"] = tuple(float(c) for c in sky)
        d["camera"] = self.camera
        return d


def define_scene(callback) -> dict:
    """dsl.define_scene: runs callback(builder) and flattens the result."""
    b = Builder()
    callback(b)
    return b.build_scene()
