"""Parity on the reference's own image-test scenes (GPU).

Every scene of the reference's image tests that this path can render
(tests/golden/ref_scenes.py restates test_box.lua, test_simple.lua and
test_bsdf.lua: triangles, cubes, spheres, disks, area / point / directional /
infinite lights, pinhole / orthographic / thin-lens cameras, Lambert,
Oren-Nayar, Phong, mirror and dielectric materials) is rendered on the GPU
and checked twice:

1. against the reference's current code on the same scene (two independent
   halves rendered here by the compiled reference, stored as 16x16 block
   means): the channel means must agree within their standard error and the
   per-block chi-square ratios of tests/ptcheck.py must stay near 1;
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

# Bounds (tests/ptcheck.py compare_blocks):
#   mean_z  channel-mean difference over its standard error: |z| > 4.5 has
#           probability ~1e-5 without bias; a planted 1 % bias of every fixture
#           scene gives |z| >= 5.2 at these sample counts (the CPU test below)
#   Xmed    median over blocks of the squared difference over the block's
#           noise estimate: ~0.6-0.9 without bias; caustics and fireflies that
#           the GPU's rounding sends elsewhere cannot move it
#   X       the summed ratio, heavy-tailed (a few nearly deterministic blocks
#           at the edges of directly seen lights carry tiny noise
#           estimates), so only a loose cap
Z_MAX = 4.5
XMED_MAX = 1.5
X_MAX = 10.0
MEAN_REL_MAX = 0.02


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
    ref_mean = np.asarray(FIX[name + "/rb0"], np.float64).mean(axis=(0, 1))
    lit = ref_mean > 1e-4
    ours_mean = np.mean([h.reshape(-1, 3).mean(0) for h in halves], axis=0)
    assert np.all(ours_mean[~lit] < 1e-4), (name, ours_mean, ref_mean)
    if lit.any():
        assert np.all(np.abs(r["mean_z"][lit]) < Z_MAX), (name, r)
        assert r["Xmed"] < XMED_MAX, (name, r)
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
@pytest.mark.parametrize("name", NAMES)
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


def test_statistics_flag_a_planted_bias():
    """CPU: the checks above reject the reference's own render scaled by 1 %
    (a mistake planted in the reference side) on every lit fixture scene, and
    accept its two halves swapped."""
    if FIX is None:
        pytest.skip("fixture missing")
    for name in NAMES:
        a0, a1 = (np.asarray(FIX[name + k], np.float64) for k in ("/rb0", "/rb1"))
        lit = a0.mean(axis=(0, 1)) > 1e-4
        if not lit.any():
            continue
        bad = ptcheck.compare_blocks(a0 * 1.01, a1 * 1.01, a0, a1)
        assert np.any(np.abs(bad["mean_z"][lit]) >= Z_MAX), (name, bad)
        same = ptcheck.compare_blocks(a1, a0, a0, a1)
        assert np.all(np.abs(same["mean_z"][lit]) < Z_MAX) and same["Xmed"] < XMED_MAX
