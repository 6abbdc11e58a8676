"""The light tracer's path code compiled for the host (CPU, no GPU needed)
against the reference's LightRenderer compiled from its sources
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

CASES = {c["name"]: c for c in ref_scenes.CASES}
SIZE, SPP = 96, 16


def _params(d, case, seed, spp=SPP):
    import dort_b200 as db
    return db.render_params(d["camera"], SIZE, SIZE, spp, min_depth=case["min_depth"],
                            max_depth=case["max_depth"], seed=seed, renderer="lt")


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("name", ["box_diff_area_pin", "box_diff_poin_pin", "box_diff_dire_pin",
                                  "box_diff_area_thin", "simple_sphe_glos_area_fwd_pin",
                                  "simple_disk_diff_mixd_2_pin"])
def test_host_light_tracer_matches_reference(name):
    import dort_b200 as db
    case = CASES[name]
    d = ref_scenes.build(case)
    ours = [ptcheck.block_means(db.host_check_render(d, _params(d, case, s)).astype(np.float64),
                                block=8) for s in (11, 12)]
    # one reference render of 4x the samples (its light tracer ignores the
    # seed: jobs are seeded by their index, light_renderer.cpp:29-31)
    ref = ptcheck.block_means(pyoracle.ref_scene_render(d, _params(d, case, 1, 4 * SPP))[0]
                              .astype(np.float64), block=8)
    r = ptcheck.compare_single(ours[0], ours[1], ref, 0.5)
    lit = ref.mean(axis=(0, 1)) > 1e-4
    assert lit.any()
    assert np.all(np.abs(r["mean_z"][lit]) < 4.5), (name, r)
    assert r["Xmed"] < 1.5, (name, r)


def test_host_light_tracer_whole_frames_only():
    import dort_b200 as db
    case = CASES["box_diff_area_pin"]
    d = ref_scenes.build(case)
    with pytest.raises(db.DortError, match="whole frames"):
        db.host_check_render(d, _params(d, case, 1), rows=(0, 10))
