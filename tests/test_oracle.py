"""Pins the oracle: the C restatement (oracle/raycast.c) reproduces the
reference's own outputs exactly -- against the committed golden vectors made
by the compiled reference (tests/golden/gen_golden.py), and against the
compiled reference directly when oracle/_ref is present."""
import os

import numpy as np
import pytest

from dort_b200 import scenes
from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "raycast_golden.npz")
CASES = ("soup", "cornell", "degenerate")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("split", ("middle", "sah"))
def test_oracle_matches_golden(golden, case, split):
    v, t, rays = golden[f"{case}_verts"], golden[f"{case}_tris"], golden[f"{case}_rays"]
    ob = po.OracleBvh(v, t, split)
    prim, tb, nodes, tests = ob.raycast(rays, counts=True)
    tb[prim == 0xFFFFFFFF] = 0.0
    assert np.array_equal(prim, golden[f"{case}_{split}_prim"])
    assert np.array_equal(tb.view(np.uint32), golden[f"{case}_{split}_tb"].view(np.uint32))
    # same traversal: the same triangle tests in the same number
    assert np.array_equal(tests, golden[f"{case}_{split}_tests"])
    anyh, _ = ob.raycast(rays, any_hit=True)
    assert np.array_equal(anyh, golden[f"{case}_{split}_any"])


def test_golden_has_hits_and_misses(golden):
    for case in CASES:
        p = golden[f"{case}_sah_prim"]
        assert 0.1 < (p != 0xFFFFFFFF).mean() < 0.95


@pytest.mark.skipif(not po.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("n,split,seed", [(2000, "sah", 1), (2000, "middle", 2),
                                          (60000, "sah", 3), (60000, "middle", 4)])
def test_oracle_matches_compiled_reference(n, split, seed):
    v, t = scenes.random_triangles(n, seed=seed)
    rb = po.RefBvh(v, t, split, threads=4)
    ob = po.OracleBvh(v, t, split)
    side = 120
    rays = np.concatenate([scenes.pinhole_rays(side, side),
                           scenes.diffuse_rays(v, t, 20000, lambda r: ob.raycast(r), seed)])
    p1, tb1, _, tests1 = ob.raycast(rays, counts=True)
    p2, tb2, tests2 = rb.raycast(rays, threads=4, counts=True)
    hit = p1 != 0xFFFFFFFF
    assert np.array_equal(p1, p2)
    assert np.array_equal(tb1[hit].view(np.uint32), tb2[hit].view(np.uint32))
    assert np.array_equal(tests1, tests2)


def test_oracle_brute_force_agrees_on_soup(golden):
    v, t, rays = golden["soup_verts"], golden["soup_tris"], golden["soup_rays"]
    bp, btb = po.brute_raycast(v, t, rays)
    gp = golden["soup_sah_prim"]
    # on a random soup the reference's BVH finds the true nearest hit
    assert (bp == gp).mean() > 0.999
