"""Generates the golden ray-cast vectors in tests/golden/raycast_golden.npz.

The expected outputs come from the reference renderer itself: its own Bvh<>
build and traversal and its Triangle / TriangleUv tests (src/dort/bvh.cpp,
box.cpp, triangle.cpp), compiled from the reference sources by
oracle/Makefile into oracle/_ref/libdort_ref.so and driven through the
harness in oracle/ref/raycast_harness.cpp.

    make -C oracle ref REF=<reference tree> && python tests/golden/gen_golden.py

Cases (all seeded): a random triangle soup, the Cornell box of the
reference's test scenes, and degenerate inputs (zero-area and duplicated
triangles, all vertices in one point).  Rays mix pinhole, diffuse bounce,
axis-parallel, zero-component and finite-window rays.  Every case is
recorded for both split methods (middle = reference default, SAH).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dort_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

OUT = os.path.join(HERE, "raycast_golden.npz")


def mixed_rays(verts, tris, n, seed):
    rng = np.random.default_rng(seed)
    rb = po.RefBvh(verts, tris, "sah")
    side = int(np.sqrt(n // 3))
    lo, hi = verts.min(0), verts.max(0)
    c = 0.5 * (lo + hi)
    ext = float(np.max(hi - lo)) + 1e-3
    coh = scenes.pinhole_rays(side, side, eye=tuple(c + np.array([0.0, 0.0, -2.5 * ext])),
                              target=tuple(c))
    dif = scenes.diffuse_rays(verts, tris, n // 3, lambda r: rb.raycast(r), seed)
    m = n - len(coh) - len(dif)
    r = np.zeros((m, 8), np.float32)
    r[:, 0:3] = lo + rng.random((m, 3)) * (hi - lo)
    axis = rng.integers(0, 3, m)
    r[np.arange(m), 4 + axis] = rng.choice([-1.0, 1.0], m)
    q = m // 2
    d = rng.normal(size=(q, 3))
    d[:, 1] = 0.0
    r[:q, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3] = rng.random(m) * 0.1 * ext
    r[:, 7] = np.where(rng.random(m) < 0.5, np.inf, r[:, 3] + rng.random(m) * ext)
    return np.ascontiguousarray(np.concatenate([coh, dif, r]).astype(np.float32))


def cases():
    out = {}
    v, t = scenes.random_triangles(1500, seed=21, sigma=0.06)
    out["soup"] = (v, t, mixed_rays(v, t, 3000, 5))
    c = scenes.cornell_box()
    cam = scenes.camera_rays(c["camera"], 32, 32)
    inner = mixed_rays(c["verts"], c["tris"], 1200, 6)
    out["cornell"] = (c["verts"], c["tris"], np.concatenate([cam, inner]))
    rng = np.random.default_rng(8)
    dv = rng.random((120, 3)).astype(np.float32)
    dt = rng.integers(0, 120, (240, 3)).astype(np.uint32)
    dt[::5, 1] = dt[::5, 0]
    dt[::7] = dt[3]
    dv[::11] = dv[0]
    out["degenerate"] = (dv, dt, mixed_rays(dv, dt, 1500, 9))
    return out


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref/libdort_ref.so is missing: run make -C oracle ref")
    arrays = {}
    for name, (v, t, rays) in cases().items():
        arrays[f"{name}_verts"] = v.astype(np.float32)
        arrays[f"{name}_tris"] = t.astype(np.uint32)
        arrays[f"{name}_rays"] = rays
        for split in ("middle", "sah"):
            rb = po.RefBvh(v, t, split, threads=1)
            prim, tb, tests = rb.raycast(rays, counts=True)
            anyh, _ = rb.raycast(rays, any_hit=True)
            tb[prim == 0xFFFFFFFF] = 0.0
            arrays[f"{name}_{split}_prim"] = prim
            arrays[f"{name}_{split}_tb"] = tb
            arrays[f"{name}_{split}_tests"] = tests
            arrays[f"{name}_{split}_any"] = anyh
            print(name, split, "rays", len(rays), "hits", int((prim != 0xFFFFFFFF).sum()))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
