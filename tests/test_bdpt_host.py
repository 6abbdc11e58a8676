"""The bidirectional tracer's path code compiled for the host (CPU, no GPU
needed) against the reference's BdptRenderer compiled from its sources
(oracle/_ref/libdort_ref.so): same scenes at a small size, two independent
halves on each side, the statistics of tests/ptcheck.py."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ptcheck  # noqa: E402
import pyoracle  # noqa: E402
import ref_scenes  # noqa: E402

SIZE, SPP = 48, 48


def _params(d, case, seed, use_t1=True, spp=SPP):
    import dort_b200 as db
    return db.render_params(d["camera"], SIZE, SIZE, spp, min_depth=case["min_depth"],
                            max_depth=case["max_depth"], seed=seed, renderer="bdpt",
                            use_t1_paths=use_t1)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("name,use_t1", [
    ("box_diff_area_pin", True), ("box_diff_area_pin", False), ("box_glos_sphe_pin", True),
    ("box_delt_dire_pin", True), ("box_diff_poin_pin", True), ("openbox_glos_infi_pin", True),
    ("box_diff_area_orth_d2", True), ("box_diff_area_thin_d1", True),
    ("simple_sphe_glos_area_fwd_pin", False), ("simple_disk_diff_mixd_2_pin", True),
    ("bsdf_dielectric_1.5@square", True), ("bsdf_phong_50@square", True)])
def test_host_bdpt_matches_reference(name, use_t1):
    import dort_b200 as db
    case = ref_scenes.case_by_name(name)
    d = ref_scenes.build(case)
    bm = lambda img: ptcheck.block_means(np.asarray(img, np.float64), block=8)  # noqa: E731
    ours = [bm(db.host_check_render(d, _params(d, case, s, use_t1))) for s in (11, 12)]
    ref = [bm(pyoracle.ref_scene_render(d, _params(d, case, s, use_t1))[0]) for s in (1, 2)]
    r = ptcheck.compare_blocks(ours[0], ours[1], ref[0], ref[1])
    lit = (ref[0] + ref[1]).mean(axis=(0, 1)) > 1e-4
    assert lit.any()
    assert np.all(np.abs(r["mean_z"][lit]) < 4.5), (name, r)
    assert r["Xmed"] < 1.5, (name, r)


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference harness not built")
def test_host_bdpt_t1_paths_matter():
    """With t = 1 connections off, the bidirectional estimate of the diffuse
    box loses the light paths that reach the camera directly: the image is
    darker by far more than its noise (both sides agree on that)."""
    import dort_b200 as db
    case = ref_scenes.case_by_name("box_diff_area_pin")
    d = ref_scenes.build(case)
    on = db.host_check_render(d, _params(d, case, 3, True)).mean()
    off = db.host_check_render(d, _params(d, case, 3, False)).mean()
    assert off < 0.95 * on


def test_host_bdpt_whole_frames_and_depth_limit():
    import dort_b200 as db
    case = ref_scenes.case_by_name("box_diff_area_pin")
    d = ref_scenes.build(case)
    with pytest.raises(db.DortError, match="whole frames"):
        db.host_check_render(d, _params(d, case, 1), rows=(0, 10))
    p = db.render_params(d["camera"], 16, 16, 1, max_depth=14, renderer="bdpt")
    with pytest.raises(db.DortError, match="max_depth"):
        db.host_check_render(d, p)
