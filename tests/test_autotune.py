"""The wavefront autotuner.

CPU: the BVH-width loop of dort_b200.autotune with the native search replaced
by a fake (no device needed): it tunes every width's scene, closes each, and
returns the fastest.
GPU: the native search (dort_gpu_autotune_wavefront / _batch) on small scenes:
its choice is one of its candidates, fits the frame, and renders the same
image as the default tuning.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

_CAMERA = {"origin": (0.0, 0.0, -5.0), "right": (1.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0),
           "forward": (0.0, 0.0, 1.0), "fov": 1.0}


class _FakeScene:
    closed = 0

    def __init__(self, width):
        self.width = width

    def close(self):
        _FakeScene.closed += 1


def test_autotune_keeps_the_fastest_width(monkeypatch):
    import dort_b200 as db
    from dort_b200 import autotune as at
    monkeypatch.setattr(at, "scene_from_dict", lambda scene, bvh_width: _FakeScene(bvh_width))
    monkeypatch.setattr(at, "tune_scene", lambda sc, p, budget: {
        "tuning": {"queue_capacity": 1 << 22, "trace_block": 128, "shade_block": 128},
        "ms": 10.0 if sc.width == 4 else 12.0, "candidates": 3, "seconds": 0.1, "cut": False})
    p = db.render_params(_CAMERA, 64, 64, 16)
    best = at.autotune({"camera": _CAMERA}, p, widths=(8, 4), budget_s=1e9)
    assert best["bvh_width"] == 4 and best["ms"] == 10.0
    assert [r["bvh_width"] for r in best["table"]] == [8, 4]
    assert _FakeScene.closed == 2


@pytest.mark.gpu
def test_native_autotune_choice_renders_the_same_image(cuda):
    import dort_b200 as db
    from dort_b200 import autotune as at
    from dort_b200 import scenes
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 96, 64, 64, max_depth=8, seed=4)
    r = at.tune_scene(sc, p, budget_s=30)
    t = r["tuning"]
    assert t["trace_block"] in (64, 128, 256) and t["shade_block"] in (64, 128, 256)
    # never more slots than twice the frame's work units (4 samples each)
    assert 32 <= t["queue_capacity"] <= max(1 << 22, 2 * 96 * 64 * 16)
    assert r["candidates"] >= 9 and r["ms"] > 0
    ref, _ = sc.render(p)
    img, _ = sc.render_wavefront(p, t)
    assert np.sqrt(((img.astype(np.float64) - ref) ** 2).mean()) / ref.mean() < 2e-3


@pytest.mark.gpu
def test_native_batch_autotune(cuda):
    import dort_b200 as db
    from dort_b200 import autotune as at
    from dort_b200 import scenes
    specs = scenes.batch_jobs(count=4, seed=9, min_tris=2000, max_tris=5000, max_res=128,
                              max_spp=64)
    jobs = [(db.scene_from_dict(sd), db.render_params(sd["camera"], w, h, spp, max_depth=d,
                                                      seed=k))
            for k, (sd, w, h, spp, d) in enumerate(specs)]
    r = at.tune_batch(jobs, budget_s=30)
    assert r["tuning"]["queue_capacity"] in (1 << 21, 1 << 22, 1 << 23, 1 << 24)
    b = db.Batch(jobs, r["tuning"])
    b.render()
    for k, (sc, p) in enumerate(jobs):
        ref, _ = sc.render(p)
        img = b.image(k)
        assert np.sqrt(((img.astype(np.float64) - ref) ** 2).mean()) / ref.mean() < 2e-3
    b.close()
