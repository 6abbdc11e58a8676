"""The device BVH builds: binned SAH (top down, the host builder's bins and
costs) and Morton order + PLOC (bottom up), each followed by the
breadth-first collapse into wide nodes.

The device collapse must equal, byte for byte, the host collapse of the same
binary tree (the shared per-node code of bvh_wide.h run on both sides); every
triangle must sit in exactly one leaf; ray queries must not depend on which
builder made the tree; and the device binned-SAH tree must be as good as the
host's by the surface-area cost.
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes

pytestmark = pytest.mark.gpu


def _soup(n, seed):
    return scenes.random_triangles(n, seed=seed)


def _degenerate_cases():
    rng = np.random.default_rng(5)
    out = {}
    # every triangle identical: all Morton codes equal, all unions equal
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    out["identical"] = (np.tile(v, (300, 1)), np.arange(900, dtype=np.uint32).reshape(-1, 3))
    # coplanar (flat in z), zero extent on one axis of the centroid bounds
    p = rng.uniform(-1, 1, (600, 3)).astype(np.float32)
    p[:, 2] = 0.25
    out["coplanar"] = (p, np.arange(600, dtype=np.uint32).reshape(-1, 3))
    # points on a line (zero-area triangles)
    t = rng.uniform(0, 1, 900).astype(np.float32)
    out["collinear"] = (np.stack([t, 2 * t, -t], 1), np.arange(900, dtype=np.uint32).reshape(-1, 3))
    # widely spread scales: tiny triangles next to huge ones
    a, ta = _soup(500, 11)
    b, tb = _soup(500, 12)
    out["scales"] = (np.concatenate([a * 1e-4, b * 1e4]).astype(np.float32),
                     np.concatenate([ta, tb + len(a)]))
    return out


BUILDS = ["device", "ploc"]


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("n,width", [(1, 8), (2, 8), (3, 8), (7, 8), (100, 8), (5000, 8),
                                     (5000, 4), (5000, 2), (200000, 8)])
def test_device_collapse_equals_host_collapse(cuda, n, width, build):
    verts, tris = _soup(n, 300 + n)
    r = db.check_device_bvh(verts, tris, bvh_width=width, bvh_build=build)
    assert r["node_bytes_differ"] == 0 and r["tri_bytes_differ"] == 0, r
    assert r["each_tri_once"], r
    assert 1 <= r["depth"] <= 64


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("name", ["identical", "coplanar", "collinear", "scales"])
def test_degenerate_meshes(cuda, name, build):
    verts, tris = _degenerate_cases()[name]
    r = db.check_device_bvh(verts, tris, bvh_build=build)
    assert r["node_bytes_differ"] == 0 and r["tri_bytes_differ"] == 0, r
    assert r["each_tri_once"], r
    if name == "collinear":
        # zero-area triangles: what the triangle test reports for them is
        # rounding noise (a "hit" point need not lie in the triangle's box),
        # so which of those survive the box tests depends on the tree
        return
    # ray queries agree with the host-built tree
    rng = np.random.default_rng(9)
    n = 20000
    o = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    tgt = verts[tris[rng.integers(0, len(tris), n), 0]]
    d = tgt - o
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 4:7] = o, d
    rays[:, 7] = 1e30
    a = db.Scene(verts, tris, bvh_build=build)
    b = db.Scene(verts, tris, bvh_build="host")
    pa, ta = a.raycast(rays)
    pb, tb = b.raycast(rays)
    assert np.array_equal(pa, pb)
    hit = pa != db.MISS
    assert np.array_equal(ta[hit].view(np.uint32), tb[hit].view(np.uint32))


@pytest.mark.parametrize("build", BUILDS)
def test_queries_do_not_depend_on_the_builder(cuda, build):
    verts, tris = _soup(100000, 77)
    rays = scenes.pinhole_rays(256, 256)
    a = db.Scene(verts, tris, bvh_build=build)
    b = db.Scene(verts, tris, bvh_build="host")
    assert a.stats()["bvh_build"] == build and b.stats()["bvh_build"] == "host"
    for any_hit in (False, True):
        ra = a.raycast(rays, any_hit=any_hit)
        rb = b.raycast(rays, any_hit=any_hit)
        if any_hit:
            assert np.array_equal(ra, rb)
        else:
            assert np.array_equal(ra[0], rb[0])
            hit = ra[0] != db.MISS
            assert np.array_equal(ra[1][hit].view(np.uint32), rb[1][hit].view(np.uint32))


def test_default_build_is_the_device(cuda):
    verts, tris = _soup(1000, 5)
    assert db.Scene(verts, tris).stats()["bvh_build"] == "device"


def test_device_tree_quality_close_to_host_sah(cuda):
    """Surface-area cost of the device trees relative to the host's
    binned-SAH tree, on a random soup and on a displaced sphere: the device
    binned SAH makes the same splits up to float rounding of the bins."""
    ws = scenes.wavefront_scene(freq=60, sky_w=16, sky_h=8)
    cases = {"soup": _soup(200000, 21), "sphere": (ws["verts"], ws["tris"])}
    for name, (verts, tris) in cases.items():
        ch = db.Scene(verts, tris, bvh_build="host").bvh_cost()
        cd = db.Scene(verts, tris, bvh_build="device").bvh_cost()
        cp = db.Scene(verts, tris, bvh_build="ploc").bvh_cost()
        assert abs(cd["sah"] / ch["sah"] - 1) < 0.02, (name, cd, ch)
        assert abs(cd["nodes"] / ch["nodes"] - 1) < 0.02, (name, cd, ch)
        assert cp["sah"] <= 1.15 * ch["sah"], (name, cp, ch)


def test_device_build_reports_invalid_input_like_the_host(cuda):
    verts, tris = _soup(10, 1)
    bad = tris.copy()
    bad[3, 1] = 999
    msgs = []
    for build in ("device", "ploc", "host"):
        with pytest.raises(db.DortError) as e:
            db.Scene(verts, bad, bvh_build=build)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1] == msgs[2] and "references vertex 999" in msgs[0]
    v2 = verts.copy()
    v2[tris[2, 0], 1] = np.nan
    with pytest.raises(db.DortError, match="is not finite"):
        db.Scene(v2, tris, bvh_build="device")
