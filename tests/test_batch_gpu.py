"""Batched wavefront rendering: many scenes / resolutions / spp / depths in
one launch.  Each job draws the random numbers a single render of it would
draw, so every batch image matches the megakernel's image of that job to
float rounding."""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from tests import ptcheck

pytestmark = pytest.mark.gpu


def test_batch_matches_single_renders(cuda):
    specs = scenes.batch_jobs(count=5, seed=40, min_tris=2000, max_tris=20000, min_res=16,
                              max_res=96, min_spp=4, max_spp=24, min_depth=3, max_depth=9)
    jobs, singles = [], []
    for k, (sd, w, h, spp, depth) in enumerate(specs):
        sc = db.scene_from_dict(sd)
        p = db.render_params(sd["camera"], w, h, spp, max_depth=depth, seed=100 + k)
        jobs.append((sc, p))
        singles.append(sc.render(p)[0])
    b = db.Batch(jobs, {"queue_capacity": 4096})
    b.render()
    st = b.stats()
    assert st["error"] == 0
    assert st["samples"] == sum(w * h * spp for (_, w, h, spp, _) in specs)
    for k in range(len(jobs)):
        img = b.image(k)
        assert img.shape == singles[k].shape
        assert ptcheck.rel_rmse(img, singles[k]) < 2e-3, k
    # a second render of the same batch gives the same images
    b.render()
    for k in range(len(jobs)):
        assert ptcheck.rel_rmse(b.image(k), singles[k]) < 2e-3
    b.close()


def test_batch_mixed_materials_and_sky(cuda):
    a = scenes.cornell_variant("delt")
    e = scenes.env_test_scene()
    sa, se = db.scene_from_dict(a), db.scene_from_dict(e)
    pa = db.render_params(a["camera"], 40, 30, 12, seed=1)
    pe = db.render_params(e["camera"], 24, 36, 20, max_depth=6, seed=2)
    b = db.Batch([(sa, pa), (se, pe), (sa, pe if False else pa)])
    b.render()
    assert ptcheck.rel_rmse(b.image(0), sa.render(pa)[0]) < 2e-3
    assert ptcheck.rel_rmse(b.image(1), se.render(pe)[0]) < 2e-3
    assert ptcheck.rel_rmse(b.image(2), b.image(0)) < 2e-3


def test_batch_rejects_bad_jobs(cuda):
    """Batches render the path tracer only: a light-tracer job is refused
    (DORT_ERR_UNSUPPORTED); an out-of-range tuning field is invalid."""
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 8, 8, 2, renderer="lt")
    with pytest.raises(db.DortError) as ex:
        db.Batch([(sc, p)])
    assert ex.value.status == -5
    p = db.render_params(sd["camera"], 8, 8, 2)
    with pytest.raises(db.DortError) as ex:
        db.Batch([(sc, p)], {"stage_queues": None, "sort_rays": None, "trace_block": 48})
    assert ex.value.status == -1 and "block sizes" in str(ex.value)
