"""Ray-cast parity on the GPU, through the C ABI, against the oracle.

Bar: nearest-hit triangle index bit-exact and (t, b1, b2) bit-identical on the
same triangle; the only accepted differences are classified exact-t ties and
hits the reference's own slab test culls (confirmed per ray).  Any-hit must
agree exactly.
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from oracle import pyoracle as po
from tests.raycheck import MISS, classify, mt_batch

pytestmark = pytest.mark.gpu


def _rays_for(verts, tris, n, seed):
    ob = po.OracleBvh(verts, tris, "sah")
    side = max(2, int(np.sqrt(n // 2)))
    coh = scenes.pinhole_rays(side, side)
    dif = scenes.diffuse_rays(verts, tris, n - len(coh), lambda r: ob.raycast(r), seed)
    return ob, np.ascontiguousarray(np.concatenate([coh, dif]))


@pytest.mark.parametrize("build", ["device", "host"])
@pytest.mark.parametrize("n_tris,n_rays,width", [
    (1, 500, 8), (16, 4000, 8), (2000, 20000, 8), (2000, 20000, 4),
    (2000, 20000, 2), (100000, 200000, 8)])
def test_random_soup_matches_oracle(cuda, n_tris, n_rays, width, build):
    verts, tris = scenes.random_triangles(n_tris, seed=100 + n_tris)
    ob, rays = _rays_for(verts, tris, n_rays, seed=7)
    ref_prim, ref_tb = ob.raycast(rays)
    sc = db.Scene(verts, tris, bvh_width=width, bvh_build=build)
    assert sc.stats()["bvh_build"] == build
    prim, tb = sc.raycast(rays)
    same, ties, box_miss, bugs = classify(verts, tris, rays, prim, tb, ref_prim, ref_tb)
    assert bugs == [], f"{len(bugs)} unexplained differences, e.g. rays {bugs[:5]}"
    assert len(ties) + len(box_miss) <= max(2, n_rays // 100000)
    ref_any, _ = ob.raycast(rays, any_hit=True)
    got_any = sc.raycast(rays, any_hit=True)
    assert np.array_equal(got_any, ref_any)


def test_golden_cornell_rays(cuda):
    """Cornell geometry: coplanar triangles sharing edges, axis-aligned walls
    and pixel-centre rays, the case where exact-t ties occur."""
    c = scenes.cornell_box()
    verts, tris = c["verts"], c["tris"]
    rays = scenes.camera_rays(c["camera"], 64, 64)
    ob = po.OracleBvh(verts, tris, "middle")
    ref_prim, ref_tb = ob.raycast(rays)
    sc = db.Scene(verts, tris)
    prim, tb = sc.raycast(rays)
    same, ties, box_miss, bugs = classify(verts, tris, rays, prim, tb, ref_prim, ref_tb)
    assert bugs == []
    assert (ref_prim != MISS).mean() > 0.9


def test_empty_scene_all_miss(cuda):
    sc = db.Scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    rays = scenes.pinhole_rays(8, 8)
    prim, _ = sc.raycast(rays)
    assert (prim == MISS).all()
    assert (sc.raycast(rays, any_hit=True) == 0).all()


def test_axis_parallel_and_windowed_rays(cuda):
    verts, tris = scenes.random_triangles(3000, seed=9, sigma=0.05)
    rng = np.random.default_rng(3)
    n = 6000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.random((n, 3)) * 1.4 - 0.2
    axis = rng.integers(0, 3, n)
    sign = rng.choice([-1.0, 1.0], n)
    rays[np.arange(n), 4 + axis] = sign               # exactly axis-parallel
    half = n // 2
    d = rng.normal(size=(half, 3))
    d[:, 0] = 0.0                                      # zero component, not axis
    rays[:half, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = rng.random(n) * 0.3                   # t_min window
    rays[:, 7] = rays[:, 3] + rng.random(n) * 0.8      # finite t_max
    rays[::17, 7] = rays[::17, 3] - 0.1                # empty window
    ob = po.OracleBvh(verts, tris, "sah")
    ref_prim, ref_tb = ob.raycast(rays)
    brute_prim, _ = po.brute_raycast(verts, tris, rays)
    sc = db.Scene(verts, tris)
    prim, tb = sc.raycast(rays)
    same, ties, box_miss, bugs = classify(verts, tris, rays, prim, tb, ref_prim, ref_tb)
    assert bugs == []
    # every box-miss of the reference is a real nearer hit
    assert all(prim[i] == brute_prim[i] for i in box_miss)
    assert np.array_equal(sc.raycast(rays, any_hit=True) != 0, brute_prim != MISS)


def test_degenerate_triangles(cuda):
    rng = np.random.default_rng(5)
    v = rng.random((300, 3)).astype(np.float32)
    tris = rng.integers(0, 300, (400, 3)).astype(np.uint32)
    tris[::5, 1] = tris[::5, 0]                        # zero-area triangles
    tris[::7] = tris[3]                                # duplicated triangles
    rays = scenes.pinhole_rays(80, 80)
    ob = po.OracleBvh(v, tris, "sah")
    ref_prim, ref_tb = ob.raycast(rays)
    sc = db.Scene(v, tris)
    prim, tb = sc.raycast(rays)
    same, ties, box_miss, bugs = classify(v, tris, rays, prim, tb, ref_prim, ref_tb)
    assert bugs == []
    # duplicates tie exactly: this build keeps the larger index
    for i in ties:
        assert prim[i] > ref_prim[i] or ref_prim[i] == MISS


def test_device_pointer_entry_matches_host_entry(cuda):
    import torch
    verts, tris = scenes.random_triangles(5000, seed=11)
    ob, rays = _rays_for(verts, tris, 10000, seed=3)
    sc = db.Scene(verts, tris)
    prim_h, tb_h = sc.raycast(rays)
    d_rays = torch.from_numpy(rays).to(cuda)
    d_prim = torch.zeros(len(rays), dtype=torch.int32, device=cuda)
    d_tb = torch.zeros((len(rays), 3), dtype=torch.float32, device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    sc.raycast_device(d_rays.data_ptr(), len(rays), d_prim.data_ptr(), d_tb.data_ptr(),
                      stream=stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_prim.cpu().numpy().view(np.uint32), prim_h)
    hit = prim_h != MISS
    assert np.array_equal(d_tb.cpu().numpy()[hit].view(np.uint32), tb_h[hit].view(np.uint32))


def test_full_size_raycast_workload(cuda):
    """1M-triangle soup, 16M rays (the benchmark workload): every reported hit
    reproduces the reference arithmetic bit-exactly, any-hit agrees with
    closest-hit on all rays, and a 1/64 subsample matches the oracle."""
    import torch
    verts, tris = scenes.random_triangles(1_000_000, seed=1)
    sc = db.Scene(verts, tris)
    cast = lambda r: sc.raycast(r)
    half = 8 * 1024 * 1024
    coh = scenes.pinhole_rays(4096, 2048)
    dif = scenes.diffuse_rays(verts, tris, half, cast, seed=2)
    rays = np.ascontiguousarray(np.concatenate([coh, dif]))
    prim, tb = sc.raycast(rays)
    hit = prim != MISS
    assert hit.mean() > 0.3
    ok, t, b1, b2 = mt_batch(verts, tris, rays[hit], prim[hit])
    assert ok.all()
    assert np.array_equal(t.view(np.uint32), tb[hit, 0].view(np.uint32))
    assert np.array_equal(b1.view(np.uint32), tb[hit, 1].view(np.uint32))
    assert np.array_equal(b2.view(np.uint32), tb[hit, 2].view(np.uint32))
    anyh = sc.raycast(rays, any_hit=True)
    assert np.array_equal(anyh != 0, hit)
    sub = rays[::64]
    ob = po.OracleBvh(verts, tris, "sah")
    ref_prim, ref_tb = ob.raycast(sub)
    same, ties, box_miss, bugs = classify(verts, tris, sub, prim[::64], tb[::64], ref_prim, ref_tb)
    assert bugs == []
    assert len(ties) + len(box_miss) <= 4


@pytest.mark.parametrize("case", ("soup", "cornell", "degenerate"))
def test_gpu_against_reference_golden(cuda, case):
    """The committed vectors produced by the compiled reference itself."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "raycast_golden.npz"))
    v, t, rays = g[f"{case}_verts"], g[f"{case}_tris"], g[f"{case}_rays"]
    sc = db.Scene(v, t)
    prim, tb = sc.raycast(rays)
    tb[prim == MISS] = 0.0
    for split in ("middle", "sah"):
        same, ties, box_miss, bugs = classify(v, t, rays, prim, tb, g[f"{case}_{split}_prim"],
                                              g[f"{case}_{split}_tb"])
        assert bugs == []
        assert len(box_miss) == 0 or case != "soup"
    anyh = sc.raycast(rays, any_hit=True)
    # any-hit can only differ where the reference's slab test culls a hit
    assert (anyh != g[f"{case}_sah_any"]).sum() <= 2
