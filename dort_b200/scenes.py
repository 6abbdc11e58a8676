"""Seeded synthetic workloads for the ray-cast and path-tracing paths.

All inputs are generated from seeds; nothing is read from disk.  The sizes
and distributions follow the benchmark configurations of the reference
project's hot path:

* ``random_triangles`` -- triangle soup: v0 ~ U[0,1]^3, v1 = v0 + N(0, s)^3,
  v2 = v0 + N(0, s)^3 (the ray-cast workload uses 1M triangles, s = 0.01).
* ``pinhole_rays`` -- coherent primary rays through pixel centres of a
  pinhole camera outside the unit cube looking at its centre.
* ``diffuse_rays`` -- secondary rays leaving the first hits of a second
  pinhole pass, cosine-distributed about the geometric normal (turned to face
  the incoming ray), with t_min = 1e-3 * t_hit as the reference's ray epsilon
  (triangle.cpp:155).

Ray layout everywhere: 8 float32 per ray = (orig.xyz, t_min, dir.xyz, t_max).
"""
from __future__ import annotations

import numpy as np

RAY_FLOATS = 8


def random_triangles(n: int, seed: int = 1, sigma: float = 0.01):
    """Returns (verts [3n,3] f32, tris [n,3] u32)."""
    rng = np.random.default_rng(seed)
    v0 = rng.random((n, 3), dtype=np.float32)
    v1 = v0 + rng.normal(0.0, sigma, (n, 3)).astype(np.float32)
    v2 = v0 + rng.normal(0.0, sigma, (n, 3)).astype(np.float32)
    verts = np.stack([v0, v1, v2], axis=1).reshape(-1, 3).astype(np.float32)
    tris = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return verts, tris


def _look_at_basis(eye, target, up=(0.0, 1.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    return eye, fwd, right, upv


def pinhole_rays(width: int, height: int, eye=(0.5, 0.5, -1.6),
                 target=(0.5, 0.5, 0.5), fov_deg: float = 40.0,
                 t_max: float = np.inf):
    """Primary rays through the pixel centres, row-major, normalized dirs."""
    eye, fwd, right, upv = _look_at_basis(eye, target)
    tan_h = np.tan(np.radians(fov_deg) * 0.5)
    aspect = width / height
    xs = ((np.arange(width, dtype=np.float64) + 0.5) / width * 2.0 - 1.0) * tan_h * aspect
    ys = (1.0 - (np.arange(height, dtype=np.float64) + 0.5) / height * 2.0) * tan_h
    rays = np.empty((height, width, RAY_FLOATS), np.float32)
    for row in range(height):
        d = fwd[None, :] + xs[:, None] * right[None, :] + ys[row] * upv[None, :]
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rays[row, :, 0:3] = eye.astype(np.float32)
        rays[row, :, 3] = 0.0
        rays[row, :, 4:7] = d.astype(np.float32)
        rays[row, :, 7] = t_max
    return rays.reshape(-1, RAY_FLOATS)


def hit_frames(verts, tris, rays, prim, tb):
    """Hit point (barycentric, as triangle.cpp:156) and unit geometric normal
    (cross(e2, e1), triangle.cpp:157) facing the incoming ray, for hit rays."""
    hit = prim != 0xFFFFFFFF
    p = prim[hit]
    t = tris[p]
    p0, p1, p2 = verts[t[:, 0]], verts[t[:, 1]], verts[t[:, 2]]
    b1 = tb[hit, 1:2]
    b2 = tb[hit, 2:3]
    b0 = np.float32(1.0) - b1 - b2
    pos = (b0 * p0 + b1 * p1 + b2 * p2).astype(np.float32)
    n = np.cross(p2 - p0, p1 - p0).astype(np.float64)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    d = rays[hit, 4:7].astype(np.float64)
    flip = np.sum(n * d, axis=1) > 0.0
    n[flip] = -n[flip]
    return hit, pos, n, tb[hit, 0]


def cosine_dirs(normals, rng):
    """Cosine-weighted directions about the given unit normals (Malley)."""
    m = len(normals)
    u1 = rng.random(m)
    u2 = rng.random(m)
    r = np.sqrt(u1)
    phi = 2.0 * np.pi * u2
    lx, ly = r * np.cos(phi), r * np.sin(phi)
    lz = np.sqrt(np.maximum(0.0, 1.0 - u1))
    # orthonormal frame per normal (Duff et al. 2017 branchless basis)
    nz = normals
    sign = np.where(nz[:, 2] >= 0.0, 1.0, -1.0)
    a = -1.0 / (sign + nz[:, 2])
    b = nz[:, 0] * nz[:, 1] * a
    t = np.stack([1.0 + sign * nz[:, 0] ** 2 * a, sign * b, -sign * nz[:, 0]], 1)
    bt = np.stack([b, sign + nz[:, 1] ** 2 * a, -nz[:, 1]], 1)
    d = lx[:, None] * t + ly[:, None] * bt + lz[:, None] * nz
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def diffuse_rays(verts, tris, count: int, cast, seed: int = 2,
                 eye=(-1.2, 1.9, -0.9), width: int | None = None):
    """``count`` diffuse bounce rays.  ``cast(rays) -> (prim, tb)`` is the
    closest-hit caster used for the second pinhole pass (any exact caster
    gives the same rays)."""
    rng = np.random.default_rng(seed)
    parts = []
    have = 0
    side = width or int(np.ceil(np.sqrt(count * 1.15)))
    # Sparse scenes may not yield enough first hits: a bounded number of
    # passes, then the hits found so far are reused with fresh directions.
    for attempt in range(4):
        if have >= count:
            break
        src = pinhole_rays(side, side, eye=eye, fov_deg=28.0 + attempt)
        prim, tb = cast(src)
        hit, pos, n, t = hit_frames(verts, tris, src, prim, tb)
        if len(pos) == 0:
            break
        reps = 1 if attempt < 3 else int(np.ceil((count - have) / len(pos)))
        pos, n, t = np.repeat(pos, reps, 0), np.repeat(n, reps, 0), np.repeat(t, reps)
        d = cosine_dirs(n, rng)
        r = np.empty((len(pos), RAY_FLOATS), np.float32)
        r[:, 0:3] = pos
        r[:, 3] = np.abs(np.float32(1e-3) * t)
        r[:, 4:7] = d.astype(np.float32)
        r[:, 7] = np.inf
        parts.append(r)
        have += len(r)
    if have < count:
        # no surface visible at all: random rays through the unit cube
        m = count - have
        r = np.empty((m, RAY_FLOATS), np.float32)
        r[:, 0:3] = rng.random((m, 3))
        r[:, 3] = 0.0
        dd = rng.normal(size=(m, 3))
        r[:, 4:7] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
        r[:, 7] = np.inf
        parts.append(r)
    return np.ascontiguousarray(np.concatenate(parts)[:count])


def raycast_workload(n_tris: int, n_rays: int, seed_tris: int = 1,
                     seed_rays: int = 2, cast_factory=None):
    """The ray-cast workload: half coherent pinhole rays (pixel centres of a
    w x h image with w = 2h), half diffuse bounce rays.  ``cast_factory(verts,
    tris)`` returns a closest-hit caster for the diffuse pass."""
    verts, tris = random_triangles(n_tris, seed_tris)
    half = n_rays // 2
    h = max(1, int(np.sqrt(half / 2)))
    w = max(1, half // h)
    coherent = pinhole_rays(w, h)
    cast = cast_factory(verts, tris)
    diffuse = diffuse_rays(verts, tris, n_rays - len(coherent), cast, seed_rays)
    rays = np.ascontiguousarray(np.concatenate([coherent, diffuse]))
    return verts, tris, rays


# ---- cameras -----------------------------------------------------------------

def look_at_camera(eye, look, up, fov: float, flip_y: bool = True):
    """Pinhole camera as dort.camera.make_pinhole with transform
    look_at(eye, look, up) * scale(1, -1, 1) (transform.cpp:146-162): returns
    {"origin", "right", "up", "forward", "fov"} with the columns of the
    camera-to-world matrix (the y column already flipped)."""
    f32 = np.float32
    eye = np.asarray(eye, f32)
    d = np.asarray(look, f32) - eye
    d = d / np.linalg.norm(d)
    upn = np.asarray(up, f32) / np.linalg.norm(np.asarray(up, f32))
    right = np.cross(upn, d)
    right = right / np.linalg.norm(right)
    upv = np.cross(d, right)
    if flip_y:
        upv = -upv
    return {"origin": eye.astype(f32), "right": right.astype(f32), "up": upv.astype(f32),
            "forward": d.astype(f32), "fov": float(fov)}


def camera_rays(cam, width: int, height: int):
    """Pixel-centre rays of PinholeCamera::sample_ray_importance
    (pinhole_camera.cpp:13-31), t in [0, inf)."""
    f32 = np.float32
    proj = f32(2.0) * f32(np.tan(0.5 * cam["fov"]))
    xs = (np.arange(width, dtype=f32) + f32(0.5)) / f32(width) - f32(0.5)
    ys = (np.arange(height, dtype=f32) + f32(0.5)) / f32(height) - f32(0.5)
    X, Y = np.meshgrid(xs, ys)
    if width > height:
        Y = Y * f32(height) / f32(width)
    else:
        X = X * f32(width) / f32(height)
    px, py = X * proj, Y * proj
    d = (px[..., None] * cam["right"] + py[..., None] * cam["up"] + cam["forward"]).astype(f32)
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.zeros((height, width, 8), f32)
    rays[..., 0:3] = cam["origin"]
    rays[..., 4:7] = d
    rays[..., 7] = np.inf
    return rays.reshape(-1, 8)


# ---- Cornell box ---------------------------------------------------------------

def _cube_tris():
    """Unit cube [-1, 1]^3 (cube_shape.cpp) as 12 triangles, normals
    cross(e2, e1) pointing outward."""
    c = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64)
    faces = []
    for a in range(3):
        for s in (-1, 1):
            idx = [i for i in range(8) if c[i, a] == s]
            # order the 4 corners around the face
            b, cc = [k for k in range(3) if k != a]
            ang = np.arctan2(c[idx, cc], c[idx, b])
            idx = [idx[k] for k in np.argsort(ang)]
            for tri in ((idx[0], idx[1], idx[2]), (idx[0], idx[2], idx[3])):
                p0, p1, p2 = c[list(tri)]
                n = np.cross(p2 - p0, p1 - p0)
                if np.dot(n, p0) < 0:
                    tri = (tri[0], tri[2], tri[1])
                faces.append(tri)
    return c, np.array(faces, np.uint32)


def _rot_y(angle):
    # rotate_y (transform.cpp:105-115)
    cs, sn = np.cos(angle), np.sin(angle)
    return np.array([[cs, 0.0, sn], [0.0, 1.0, 0.0], [-sn, 0.0, cs]])


def cornell_box(white=(0.75, 0.75, 0.75), red=(0.63, 0.06, 0.05),
                green=(0.14, 0.45, 0.09), light_radiance=(17.0, 12.0, 4.0),
                light_size=0.5):
    """The Cornell box of the reference's test scenes (test/test_box.lua:40-105,
    scale s = 0.01): 10 wall triangles, two rotated boxes (12 triangles each)
    and a light_size^2 quad light (2 emissive triangles) just below the
    ceiling.  Materials: 0 white, 1 red, 2 green, 3 black (light)."""
    s = 0.01
    P = np.array([[552.8, 0, 0], [0, 0, 0], [0, 0, 559.2], [549.6, 0, 559.2],
                  [556, 548.8, 0], [556, 548.8, 559.2], [0, 548.8, 559.2], [0, 548.8, 0]],
                 np.float64) * s
    V = [0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7, 6, 5, 3, 6, 3, 2, 7, 6, 2, 7, 2, 1,
         0, 3, 5, 0, 5, 4]
    verts = [P]
    tris = [np.array(V, np.uint32).reshape(-1, 3)]
    # floor, ceiling, back wall: white; left wall (x = 0): green; right: red
    mats = [0, 0, 0, 0, 0, 0, 2, 2, 1, 1]
    cube_v, cube_t = _cube_tris()
    for trans, ang, scl in (((185, 82.5, 169), -0.29, (165 / 2, 165 / 2, 165 / 2)),
                            ((368, 165, 351), -1.27, (165 / 2, 330 / 2, 165 / 2))):
        v = (cube_v * (np.array(scl) * s)) @ _rot_y(ang).T + np.array(trans) * s
        tris.append(cube_t + sum(len(x) for x in verts))
        verts.append(v)
        mats += [0] * 12
    cx, cz, y = 278 * s, 279.5 * s, 548.8 * s - 1 * s
    h = light_size / 2
    L = np.array([[cx + h, y, cz - h], [cx + h, y, cz + h], [cx - h, y, cz + h],
                  [cx - h, y, cz - h]])
    base = sum(len(x) for x in verts)
    verts.append(L)
    tris.append(np.array([[2, 1, 0], [3, 2, 0]], np.uint32) + base)
    mats += [3, 3]
    verts = np.concatenate(verts).astype(np.float32)
    tris = np.concatenate(tris).astype(np.uint32)
    emission = np.zeros((len(tris), 3), np.float32)
    emission[-2:] = light_radiance
    materials = [
        {"kind": 0, "color": white}, {"kind": 0, "color": red},
        {"kind": 0, "color": green}, {"kind": 0, "color": (0.0, 0.0, 0.0)},
    ]
    cam = look_at_camera((278 * s, 273 * s, -800 * s), (278 * s, 273 * s, 0.0),
                         (0.0, 1.0, 0.0), 0.686)
    return {"verts": verts, "tris": tris, "tri_material": np.array(mats, np.uint32),
            "materials": materials, "tri_emission": emission, "camera": cam}


def cornell_variant(kind: str = "diff", light: str = "area"):
    """Cornell box variants after the reference's test scenes
    (test/test_box.lua:110-140): "diff" all Lambert, "glos" Phong boxes and
    right wall, "delt" mirror right box + glass left box + mirror left wall;
    light "area" (quad light), "infi" (constant sky, open box) or "both"."""
    c = cornell_box()
    mats = c["materials"]
    if kind == "glos":
        # phong_material { albedo = a, exponent = 50 }: glossy albedo
        # defaults to the diffuse one (lua_material.cpp:166-176)
        mats.append({"kind": 3, "color": (0.5, 0.5, 0.5), "color2": (0.5, 0.5, 0.5),
                     "param": (50.0,)})
        mats.append({"kind": 3, "color": (0.5, 0.0, 0.0), "color2": (0.5, 0.0, 0.0),
                     "param": (50.0,)})
        tm = c["tri_material"]
        tm[10:34] = len(mats) - 2          # both boxes glossy white
        tm[8:10] = len(mats) - 1           # right wall glossy red
    elif kind == "delt":
        mats.append({"kind": 1, "color": (1.0, 1.0, 1.0)})
        mats.append({"kind": 2, "color": (1.0, 1.0, 1.0), "color2": (1.0, 1.0, 1.0),
                     "param": (1.3,)})
        tm = c["tri_material"]
        tm[22:34] = len(mats) - 2          # right box mirror
        tm[10:22] = len(mats) - 1          # left box glass
        tm[6:8] = len(mats) - 2            # left wall mirror
    if light in ("infi", "both"):
        c["sky_const"] = (1.0, 1.0, 1.0)
    if light == "infi":
        c["tri_emission"] = np.zeros_like(c["tri_emission"])
        # open box: drop the back wall so the sky is visible
        keep = np.ones(len(c["tris"]), bool)
        keep[4:6] = False
        c["tris"] = c["tris"][keep]
        c["tri_material"] = c["tri_material"][keep]
        c["tri_emission"] = c["tri_emission"][keep]
    return c


def procedural_sky(width: int = 256, height: int = 128, seed: int = 3):
    """Latitude-longitude HDR sky (row 0 = zenith): a vertical gradient plus a
    sun lobe; float32 [height, width, 3]."""
    v = (np.arange(height, dtype=np.float64) + 0.5) / height          # theta / pi
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    theta = v * np.pi
    phi = (u - 0.5) * 2.0 * np.pi
    T, P = np.meshgrid(theta, phi, indexing="ij")
    up = np.cos(T)
    sky = np.stack([0.35 + 0.5 * np.clip(up, 0, 1), 0.45 + 0.55 * np.clip(up, 0, 1),
                    0.7 + 0.6 * np.clip(up, 0, 1)], -1)
    ground = np.array([0.25, 0.22, 0.2])
    sky = np.where(up[..., None] < 0.0, ground, sky)
    rng = np.random.default_rng(seed)
    sun_t, sun_p = 0.3 + 0.1 * rng.random(), (rng.random() - 0.5) * np.pi
    d = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1)
    s = np.array([np.sin(sun_t) * np.cos(sun_p), np.cos(sun_t), np.sin(sun_t) * np.sin(sun_p)])
    cosang = d @ s
    sun = 40.0 * np.exp((cosang - 1.0) * 400.0)
    sky = sky + sun[..., None] * np.array([1.0, 0.9, 0.7])
    return sky.astype(np.float32)


def env_test_scene(seed: int = 11, conductor: bool = False):
    """A small scene lit only by the procedural sky: a ground quad and a few
    random boxes of Lambert / mirror / glass / Phong (/ GGX conductor, which
    has no reference counterpart, when ``conductor``)."""
    rng = np.random.default_rng(seed)
    verts = [np.array([[-3, 0, -3], [3, 0, -3], [3, 0, 3], [-3, 0, 3]], np.float64)]
    tris = [np.array([[0, 2, 1], [0, 3, 2]], np.uint32)]
    mats = [0, 0]
    cube_v, cube_t = _cube_tris()
    for k in range(6):
        sc = 0.25 + 0.3 * rng.random(3)
        pos = np.array([rng.uniform(-1.8, 1.8), sc[1], rng.uniform(-1.8, 1.8)])
        v = (cube_v * sc) @ _rot_y(rng.uniform(0, 3)).T + pos
        tris.append(cube_t + sum(len(x) for x in verts))
        verts.append(v)
        mats += [1 + k % 5] * 12
    materials = [
        {"kind": 0, "color": (0.6, 0.6, 0.6)},
        {"kind": 0, "color": (0.7, 0.3, 0.2)},
        {"kind": 1, "color": (0.9, 0.9, 0.9)},
        {"kind": 2, "color": (1.0, 1.0, 1.0), "color2": (1.0, 1.0, 1.0), "param": (1.5,)},
        {"kind": 3, "color": (0.3, 0.3, 0.5), "color2": (0.4, 0.4, 0.4), "param": (30.0,)},
        {"kind": 4, "color": (0.9, 0.7, 0.4), "param": (0.2,)} if conductor
        else {"kind": 0, "color": (0.2, 0.5, 0.3)},
    ]
    cam = look_at_camera((0.0, 2.5, -6.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 0.9)
    return {"verts": np.concatenate(verts).astype(np.float32),
            "tris": np.concatenate(tris).astype(np.uint32),
            "tri_material": np.array(mats, np.uint32), "materials": materials,
            "tri_emission": None, "sky_rgb": procedural_sky(), "camera": cam}


# ---- the 1080p wavefront workload ------------------------------------------------

def _hash3(ix, iy, iz, seed):
    """Integer lattice hash -> [0, 1) (a 32-bit multiply-xorshift mix)."""
    h = (ix.astype(np.uint64) * np.uint64(73856093)) ^ (iy.astype(np.uint64) * np.uint64(19349663)) \
        ^ (iz.astype(np.uint64) * np.uint64(83492791)) ^ np.uint64(seed * 2654435761 % (1 << 32))
    h = h & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    h = (h * np.uint64(0x7FEB352D)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(0x846CA68B)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    return (h.astype(np.float64) / 4294967296.0)


def value_noise(p, seed):
    """Trilinear value noise in [-1, 1] at points p [n, 3] (smoothstep fade)."""
    f = np.floor(p)
    t = p - f
    t = t * t * (3.0 - 2.0 * t)
    i = f.astype(np.int64) + (1 << 20)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (t[:, 0] if dx else 1 - t[:, 0]) * (t[:, 1] if dy else 1 - t[:, 1]) * \
                    (t[:, 2] if dz else 1 - t[:, 2])
                out += w * _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
    return out * 2.0 - 1.0


def fbm(p, seed, octaves=6, base_freq=2.0):
    total = np.zeros(len(p))
    amp, freq, norm = 1.0, base_freq, 0.0
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed + o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def icosphere(freq: int):
    """Geodesic sphere: each icosahedron face split into freq^2 triangles,
    vertices projected to the unit sphere.  Vertices are shared within a face
    (not across faces).  Returns (verts [V,3] f64, tris [20 freq^2, 3])."""
    t = (1.0 + 5 ** 0.5) / 2.0
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 np.float64)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]])
    n = freq
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    mask = ii + jj <= n
    ii, jj = ii[mask], jj[mask]
    idx = -np.ones((n + 1, n + 1), np.int64)
    idx[ii, jj] = np.arange(len(ii))
    # local triangles of the barycentric grid
    a_i, a_j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = a_i + a_j < n
    t_up = np.stack([idx[a_i[up], a_j[up]], idx[a_i[up] + 1, a_j[up]], idx[a_i[up], a_j[up] + 1]], 1)
    dn = a_i + a_j < n - 1
    t_dn = np.stack([idx[a_i[dn] + 1, a_j[dn]], idx[a_i[dn] + 1, a_j[dn] + 1],
                     idx[a_i[dn], a_j[dn] + 1]], 1)
    local = np.concatenate([t_up, t_dn])
    npts = len(ii)
    verts, tris = [], []
    for f_i, (a, b, c) in enumerate(F):
        wa = (n - ii - jj) / n
        wb = ii / n
        wc = jj / n
        p = wa[:, None] * V[a] + wb[:, None] * V[b] + wc[:, None] * V[c]
        p /= np.linalg.norm(p, axis=1, keepdims=True)
        verts.append(p)
        tris.append(local + f_i * npts)
    return np.concatenate(verts), np.concatenate(tris).astype(np.uint32)


def wavefront_scene(freq: int = 316, sky_w: int = 1024, sky_h: int = 512, seed: int = 3,
                    n_materials: int = 96, conductor: bool = True):
    """The 1080p wavefront workload: a geodesic icosphere of frequency `freq`
    (20 freq^2 triangles; 1,997,120 at 316) displaced along the normal by fBm
    (amplitude 0.1, 6 octaves), on a 2-triangle ground plane, lit by a
    procedural sky_w x sky_h HDR sky.  Materials are a seeded mix of Lambert
    (albedo U(0.2, 0.8)), GGX conductor (alpha U(0.05, 0.5)) and dielectric
    (ior 1.5), assigned per surface patch."""
    rng = np.random.default_rng(seed)
    v, t = icosphere(freq)
    disp = 0.1 * fbm(v * 1.5, seed, octaves=6)
    v = v * (1.0 + disp)[:, None]
    v = v + np.array([0.0, 1.15, 0.0])
    # materials: table of n_materials entries, one per patch of ~256 triangles
    mats = []
    for k in range(n_materials):
        r = k % 3 if conductor else k % 2 * 2
        if r == 0:
            mats.append({"kind": 0, "color": tuple(rng.uniform(0.2, 0.8, 3))})
        elif r == 1:
            mats.append({"kind": 4, "color": tuple(rng.uniform(0.5, 0.95, 3)),
                         "param": (float(rng.uniform(0.05, 0.5)),)})
        else:
            mats.append({"kind": 2, "color": (1.0, 1.0, 1.0), "color2": (1.0, 1.0, 1.0),
                         "param": (1.5,)})
    patch = np.arange(len(t)) // 256
    tri_mat = _hash3(patch, patch * 7 + 1, patch * 13 + 2, seed) * n_materials
    tri_mat = np.minimum(tri_mat.astype(np.uint32), n_materials - 1)
    ground_v = np.array([[-20, 0, -20], [20, 0, -20], [20, 0, 20], [-20, 0, 20]], np.float64)
    ground_t = np.array([[0, 2, 1], [0, 3, 2]], np.uint32) + len(v)
    mats.append({"kind": 0, "color": (0.45, 0.42, 0.4)})
    verts = np.concatenate([v, ground_v]).astype(np.float32)
    tris = np.concatenate([t, ground_t]).astype(np.uint32)
    tri_mat = np.concatenate([tri_mat, np.full(2, len(mats) - 1, np.uint32)])
    cam = look_at_camera((0.0, 1.6, -4.2), (0.0, 1.05, 0.0), (0.0, 1.0, 0.0), 0.75)
    return {"verts": verts, "tris": tris, "tri_material": tri_mat, "materials": mats,
            "tri_emission": None, "sky_rgb": procedural_sky(sky_w, sky_h, seed), "camera": cam}


def adjoint_scene(n_tris: int = 500_000, seed: int = 5):
    """The adjoint workload: a random-triangle soup (the ray-cast generator,
    seed 5) with per-triangle RGB albedo U(0.1, 0.9), plus 8 emissive
    triangles in a ring above the soup, facing down.  Returns the scene dict
    plus "tri_albedo" and the emissive triangles' indices in "lights"."""
    rng = np.random.default_rng(seed)
    verts, tris = random_triangles(n_tris, seed=seed, sigma=0.02)
    albedo = rng.uniform(0.1, 0.9, (n_tris, 3)).astype(np.float32)
    lv, lt = [], []
    base = len(verts)
    for k in range(8):
        ang = 2 * np.pi * k / 8
        c = np.array([0.5 + 0.55 * np.cos(ang), 1.45, 0.5 + 0.55 * np.sin(ang)])
        a, b = 0.22, 0.18
        # cross(e2, e1) must point down (-y): p0, p1 = p0 + (0,0,b), p2 = p0 + (a,0,0)
        p0 = c + np.array([-a / 2, 0.0, -b / 2])
        lv += [p0, p0 + np.array([0.0, 0.0, b]), p0 + np.array([a, 0.0, 0.0])]
        lt.append([base + 3 * k, base + 3 * k + 1, base + 3 * k + 2])
    verts = np.concatenate([verts, np.array(lv, np.float32)]).astype(np.float32)
    tris = np.concatenate([tris, np.array(lt, np.uint32)]).astype(np.uint32)
    n = len(tris)
    emission = np.zeros((n, 3), np.float32)
    cols = rng.uniform(0.5, 1.0, (8, 3)) * 30.0
    emission[n_tris:] = cols
    tri_albedo = np.concatenate([albedo, np.zeros((8, 3), np.float32)])
    mats = [{"kind": 0, "color": (0.5, 0.5, 0.5)}, {"kind": 0, "color": (0.0, 0.0, 0.0)}]
    tri_mat = np.zeros(n, np.uint32)
    tri_mat[n_tris:] = 1
    cam = look_at_camera((0.5, 1.0, -1.4), (0.5, 0.45, 0.5), (0.0, 1.0, 0.0), 0.9)
    return {"verts": verts, "tris": tris, "tri_material": tri_mat, "materials": mats,
            "tri_emission": emission, "tri_albedo": tri_albedo,
            "lights": np.arange(n_tris, n, dtype=np.int64), "camera": cam}


def soup_with_light(n_tris: int, seed: int):
    """A random-triangle soup (the ray-cast generator) with Lambert albedo
    0.6 and one 2-triangle quad light above it, facing down (the batched
    workload's scene)."""
    verts, tris = random_triangles(n_tris, seed=seed, sigma=0.02)
    base = len(verts)
    L = np.array([[0.7, 1.4, 0.3], [0.7, 1.4, 0.7], [0.3, 1.4, 0.7], [0.3, 1.4, 0.3]], np.float32)
    verts = np.concatenate([verts, L]).astype(np.float32)
    # (2,1,0), (3,2,0) as the Cornell light: cross(e2, e1) points down
    lt = np.array([[base + 2, base + 1, base], [base + 3, base + 2, base]], np.uint32)
    tris = np.concatenate([tris, lt]).astype(np.uint32)
    em = np.zeros((len(tris), 3), np.float32)
    em[-2:] = (12.0, 11.0, 10.0)
    tm = np.zeros(len(tris), np.uint32)
    tm[-2:] = 1
    mats = [{"kind": 0, "color": (0.6, 0.6, 0.6)}, {"kind": 0, "color": (0.0, 0.0, 0.0)}]
    cam = look_at_camera((0.5, 0.8, -1.3), (0.5, 0.45, 0.5), (0.0, 1.0, 0.0), 0.9)
    return {"verts": verts, "tris": tris, "tri_material": tm, "materials": mats,
            "tri_emission": em, "camera": cam}


def batch_jobs(count: int = 64, seed: int = 4, min_tris: int = 10_000, max_tris: int = 500_000,
               min_res: int = 64, max_res: int = 1024, min_spp: int = 16, max_spp: int = 512,
               min_depth: int = 8, max_depth: int = 16):
    """The batched workload: `count` seeded jobs, job k a soup_with_light of
    log-uniform triangle count (seed 4 + k), resolution log-uniform per axis,
    spp uniform in [min_spp, max_spp], depth uniform in [min_depth,
    max_depth].  Returns a list of (scene dict, width, height, spp, depth)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(min_tris), np.log(max_tris))))
        w = int(np.exp(rng.uniform(np.log(min_res), np.log(max_res))))
        h = int(np.exp(rng.uniform(np.log(min_res), np.log(max_res))))
        spp = int(rng.integers(min_spp, max_spp + 1))
        depth = int(rng.integers(min_depth, max_depth + 1))
        jobs.append((soup_with_light(n, seed + k), w, h, spp, depth))
    return jobs
