"""The device traversal code compiled for the host (dort_gpu_host_check_raycast)
against the oracle: checks the wide-BVH builder, the quantization margins and
the octant-ordered traversal without a GPU."""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from oracle import pyoracle as po
from tests.raycheck import classify


@pytest.mark.parametrize("n_tris,n_rays,width", [
    (1, 300, 8), (10, 2000, 8), (300, 4000, 4), (3000, 12000, 8), (3000, 6000, 2),
    (40000, 30000, 8)])
def test_host_traversal_matches_oracle(n_tris, n_rays, width):
    verts, tris = scenes.random_triangles(n_tris, seed=n_tris)
    ob = po.OracleBvh(verts, tris, "sah")
    side = int(np.sqrt(n_rays // 2))
    rays = np.concatenate([scenes.pinhole_rays(side, side),
                           scenes.diffuse_rays(verts, tris, n_rays // 2, lambda r: ob.raycast(r), 7)])
    ref_prim, ref_tb = ob.raycast(rays)
    prim, tb, depth = db.host_check_raycast(verts, tris, rays, bvh_width=width)
    same, ties, box_miss, bugs = classify(verts, tris, rays, prim, tb, ref_prim, ref_tb)
    assert bugs == []
    assert len(ties) + len(box_miss) <= 1
    ref_any, _ = ob.raycast(rays, any_hit=True)
    got_any, _ = db.host_check_raycast(verts, tris, rays, any_hit=True, bvh_width=width)
    assert np.array_equal(got_any, ref_any)
    assert depth <= 64


def test_host_traversal_cornell_ties_classified():
    c = scenes.cornell_box()
    rays = scenes.camera_rays(c["camera"], 48, 48)
    ob = po.OracleBvh(c["verts"], c["tris"], "middle")
    ref_prim, ref_tb = ob.raycast(rays)
    prim, tb, _ = db.host_check_raycast(c["verts"], c["tris"], rays)
    same, ties, box_miss, bugs = classify(c["verts"], c["tris"], rays, prim, tb, ref_prim, ref_tb)
    assert bugs == []


def test_degenerate_inputs_host():
    rng = np.random.default_rng(5)
    v = rng.random((100, 3)).astype(np.float32)
    t = rng.integers(0, 100, (200, 3)).astype(np.uint32)
    t[::5, 1] = t[::5, 0]
    t[::7] = t[3]
    # all triangles at one point: zero extent on every axis
    v2 = np.zeros((3, 3), np.float32)
    t2 = np.tile(np.array([[0, 1, 2]], np.uint32), (50, 1))
    for verts, tris in ((v, t), (v2, t2)):
        rays = scenes.pinhole_rays(40, 40)
        ob = po.OracleBvh(verts, tris, "sah")
        ref_prim, ref_tb = ob.raycast(rays)
        prim, tb, _ = db.host_check_raycast(verts, tris, rays)
        same, ties, box_miss, bugs = classify(verts, tris, rays, prim, tb, ref_prim, ref_tb)
        assert bugs == []
