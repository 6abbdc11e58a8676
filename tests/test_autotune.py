"""CPU: the autotuner's search with the GPU frame replaced by a fake timing
(no device needed): it times every candidate that fits the proxy frame,
skips capacities far above the proxy's samples, and returns the fastest."""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


_CAMERA = {"origin": (0.0, 0.0, -5.0), "right": (1.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0),
           "forward": (0.0, 0.0, 1.0), "fov": 1.0}


class _FakeScene:
    def __init__(self, width, clock):
        self.width, self.clock = width, clock

    def render_wavefront(self, params, tuning):
        # a made-up cost: larger queues and 128-thread blocks are faster,
        # width 8 beats width 4
        ms = (100.0 / tuning["queue_capacity"] ** 0.1 + abs(tuning["trace_block"] - 128) / 64
              + abs(tuning["shade_block"] - 128) / 64 + (0.0 if self.width == 8 else 5.0))
        self.clock.append(tuning["queue_capacity"])
        return None, {"ms": ms}

    def close(self):
        pass


def test_autotune_picks_the_fastest_candidate(monkeypatch):
    import dort_b200 as db
    from dort_b200 import autotune as at
    seen = []
    monkeypatch.setattr(at, "scene_from_dict", lambda scene, bvh_width: _FakeScene(bvh_width, seen))
    d = {"camera": _CAMERA}
    p = db.render_params(d["camera"], 1920, 1080, 256, max_depth=8)
    best = at.autotune(d, p, proxy_spp=4, budget_s=1e9)
    assert best["bvh_width"] == 8
    assert best["tuning"] == {"queue_capacity": 1 << 24, "trace_block": 128, "shade_block": 128}
    assert len(best["table"]) == 2 * 3 * 3 * 3
    assert set(seen) == set(at.DEFAULT_CAPACITIES)


def test_autotune_skips_queues_far_above_the_proxy(monkeypatch):
    import dort_b200 as db
    from dort_b200 import autotune as at
    seen = []
    monkeypatch.setattr(at, "scene_from_dict", lambda scene, bvh_width: _FakeScene(bvh_width, seen))
    d = {"camera": _CAMERA}
    # 256 x 256 x 4 proxy samples: only the smallest capacity is tried
    p = db.render_params(d["camera"], 256, 256, 64, max_depth=8)
    best = at.autotune(d, p, proxy_spp=4, budget_s=1e9)
    assert set(seen) == {min(at.DEFAULT_CAPACITIES)}
    assert best["tuning"]["queue_capacity"] == min(at.DEFAULT_CAPACITIES)
