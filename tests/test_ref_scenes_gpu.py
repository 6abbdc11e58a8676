"""Parity on the reference's own image-test scenes (GPU).

Every scene of the reference's image tests that this path can render
(tests/golden/ref_scenes.py restates test_box.lua, test_simple.lua and
test_bsdf.lua: triangles, cubes, spheres, disks, area / point / directional /
infinite lights, pinhole / orthographic / thin-lens cameras, Lambert,
Oren-Nayar, Phong, mirror and dielectric materials) is rendered on the GPU
and checked twice:

1. against the reference's current code on the same scene (two independent
   halves rendered here by the compiled reference, stored as 16x16 block
   means): the block chi-square ratio X of tests/ptcheck.py must stay near 1
   and the channel means within a few percent;
2. by the reference's own acceptance test, test_convergence
   (convergence_test.cpp:10-101), against the reference's stored converged
   image: the GPU render must pass wherever the reference's current code
   passes with margin, and must fail wherever the stored image no longer
   matches the reference's code (some stored images predate changes of the
   reference; for those the reference's own render fails the same way).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import ptcheck  # noqa: E402
import ref_scenes  # noqa: E402

FIX_PATH = os.path.join(HERE, "golden", "ref_images.npz")
FIX = np.load(FIX_PATH) if os.path.exists(FIX_PATH) else None
NAMES = [str(n) for n in FIX["names"]] if FIX is not None else []
CASES = {c["name"]: c for c in ref_scenes.CASES}

# Bounds: X is 1 in expectation without bias but heavy-tailed where a few
# blocks carry almost deterministic values (the edges of directly seen lights:
# two halves of such a block barely differ, so its noise estimate is tiny);
# a bias of a few percent gives X in the tens at these sample counts.
X_MAX = 3.5
MEAN_REL_MAX = 0.02   # channel means


def _render(name, renderer):
    import dort_b200 as db
    case = CASES[name]
    d = ref_scenes.build(case)
    sc = db.scene_from_dict(d)
    spp = int(FIX["spp"])
    halves = []
    for seed in (101, 102):
        p = db.render_params(d["camera"], case["width"], case["height"], spp,
                             min_depth=case["min_depth"], max_depth=case["max_depth"],
                             sample_all_lights=case["sample_all_lights"], seed=seed)
        img = (sc.render(p) if renderer == "megakernel" else sc.render_wavefront(p))[0]
        halves.append(img.astype(np.float64))
    sc.close()
    return halves


def _check(name, halves):
    case = CASES[name]
    ob = [ptcheck.block_means(h) for h in halves]
    r = ptcheck.compare_blocks(ob[0], ob[1], FIX[name + "/rb0"], FIX[name + "/rb1"])
    lit = np.asarray(FIX[name + "/rb0"], np.float64).mean(axis=(0, 1)) > 1e-4
    assert np.all(r["X"][lit] < X_MAX), (name, r)
    assert np.all(np.abs(r["mean_rel"][lit]) < MEAN_REL_MAX), (name, r)

    full = (halves[0] + halves[1]) / 2
    worst, fail = ptcheck.reference_convergence(FIX[name + "/tmeans"], FIX[name + "/tiles"],
                                                full, variation=case["variation"])
    ref_code = float(FIX[name + "/conv"])
    if ref_code <= 0.8:
        assert worst <= 1.0, (name, worst, fail)
    elif ref_code > 1.25:
        assert worst > 1.0, (name, worst, ref_code)


@pytest.mark.gpu
@pytest.mark.skipif(FIX is None, reason="tests/golden/ref_images.npz missing")
@pytest.mark.parametrize("name", NAMES)
def test_reference_scene_megakernel(name, cuda):
    _check(name, _render(name, "megakernel"))


@pytest.mark.gpu
@pytest.mark.skipif(FIX is None, reason="tests/golden/ref_images.npz missing")
@pytest.mark.parametrize("name", [n for n in NAMES if not CASES[n]["sample_all_lights"]])
def test_reference_scene_wavefront(name, cuda):
    _check(name, _render(name, "wavefront"))


def test_reference_scene_fixture_is_consistent():
    """CPU: the fixture covers the listed cases with the expected shapes, and
    the restated scenes build."""
    if FIX is None:
        pytest.skip("fixture missing")
    assert len(NAMES) >= 80
    for name in NAMES:
        case = CASES[name]
        by, bx = (case["height"] + 15) // 16, (case["width"] + 15) // 16
        assert FIX[name + "/rb0"].shape == (by, bx, 3)
        assert FIX[name + "/tmeans"].shape[0] == FIX[name + "/tiles"].shape[0]
        d = ref_scenes.build(case)
        assert d["camera"] is not None
