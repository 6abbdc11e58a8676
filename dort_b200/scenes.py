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
