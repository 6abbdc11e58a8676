"""Helpers shared by the ray-cast parity tests: comparison against the oracle
with every disagreement classified."""
from __future__ import annotations

import numpy as np

from oracle import pyoracle as po

MISS = 0xFFFFFFFF


def classify(verts, tris, rays, got_prim, got_tb, ref_prim, ref_tb):
    """Returns (n_equal, ties, ref_box_miss, bugs) where every differing ray
    is one of:
      tie          both triangles hit at exactly the same t (the reference
                   keeps the last one it tests, this build the larger index);
      ref_box_miss this build found a strictly nearer hit that the reference's
                   non-conservative slab test culled (confirmed by testing the
                   triangle directly);
      bug          anything else.
    """
    diff = np.nonzero(got_prim != ref_prim)[0]
    ties, box_miss, bugs = [], [], []
    verts = np.asarray(verts, np.float32).reshape(-1, 3)
    tris = np.asarray(tris, np.uint32).reshape(-1, 3)
    for i in diff:
        g, r = int(got_prim[i]), int(ref_prim[i])
        ray = rays[i]
        g_ok, g_tb = (False, None) if g == MISS else po.triangle_hit(
            verts[tris[g, 0]], verts[tris[g, 1]], verts[tris[g, 2]], ray)
        r_ok, r_tb = (False, None) if r == MISS else po.triangle_hit(
            verts[tris[r, 0]], verts[tris[r, 1]], verts[tris[r, 2]], ray)
        if g_ok and r_ok and g_tb[0] == r_tb[0]:
            ties.append(i)
        elif g_ok and (not r_ok or g_tb[0] < r_tb[0]):
            box_miss.append(i)
        else:
            bugs.append(i)
    same = got_prim == ref_prim
    hit = same & (ref_prim != MISS)
    tb_bad = np.nonzero(hit & np.any(got_tb.view(np.uint32) != ref_tb.view(np.uint32), axis=1))[0]
    return int(same.sum()), ties, box_miss, list(bugs) + [int(x) for x in tb_bad]


def mt_batch(verts, tris, rays, prim):
    """Vectorized restatement of the reference Moller-Trumbore arithmetic
    (triangle.cpp:109-134) in float32 numpy (IEEE, no fused multiply-add) for
    the reported triangle of each ray: returns (ok, t, b1, b2)."""
    f = np.float32
    v = np.asarray(verts, f).reshape(-1, 3)
    t3 = np.asarray(tris, np.uint32).reshape(-1, 3)[prim]
    p0, p1, p2 = v[t3[:, 0]], v[t3[:, 1]], v[t3[:, 2]]
    o, d = rays[:, 0:3], rays[:, 4:7]
    tmin, tmax = rays[:, 3], rays[:, 7]
    e1 = p1 - p0
    e2 = p2 - p0

    def cross(a, b):
        return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                         a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                         a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)

    def dot(a, b):
        return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]

    with np.errstate(all="ignore"):
        s1 = cross(d, e2)
        det = dot(s1, e1)
        inv = f(1.0) / det
        s = o - p0
        b1 = inv * dot(s1, s)
        s2 = cross(s, e1)
        b2 = inv * dot(s2, d)
        t = inv * dot(s2, e2)
        # rejection tests as written in the reference (NaN passes them)
        ok = ~(det == 0) & ~((b1 < 0) | (b1 > 1)) & ~((b2 < 0) | ((b1 + b2) > 1)) & \
             ~((t < tmin) | (t > tmax))
    return ok, t, b1, b2
