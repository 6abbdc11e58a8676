"""The bidirectional path tracer ("bdpt" renderer) on the GPU.

1. Against the reference's own BdptRenderer (bdpt_renderer.cpp:9-468) on the
   scenes its image tests render with "bdpt" (tests/golden/bdpt_images.npz,
   two independent halves by the compiled reference): channel means within
   4.5 standard errors, median per-block chi-square ratio below 1.5 -- the
   bounds of the path tracer's parity test (tests/test_ref_scenes_gpu.py).
   With t = 1 connections off on a subset, against the reference's renders
   with use_t1_paths = false (<name>/nt0, nt1): the reference keeps those
   connections in its MIS weights, so the image without them is darker, a
   debugging switch that the GPU reproduces.
2. Against the path tracer: on the scenes where the reference's own "bdpt"
   and "pt" renders agree (its two fixtures pass these statistics against
   each other with a margin; no Phong surfaces), the GPU's bidirectional image and the reference's "pt" image
   (tests/golden/ref_images.npz) agree too -- the check the reference's
   tests make (each renderer's image against a converged "pt" image).  On
   the other scenes the reference's bidirectional tracer converges elsewhere
   (Phong surfaces 0.1-2 % darker, delta surfaces ~10 % and infinite lights
   ~3 % brighter, the thin lens through its pivot importance) and test 1
   holds the GPU to that.
3. The contract of the entry points: the bidirectional tracer renders through
   dort_gpu_render / _device only, with max_depth <= 13.
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

BD_PATH = os.path.join(HERE, "golden", "bdpt_images.npz")
PT_PATH = os.path.join(HERE, "golden", "ref_images.npz")
BD = np.load(BD_PATH) if os.path.exists(BD_PATH) else None
PT = np.load(PT_PATH) if os.path.exists(PT_PATH) else None
NAMES = [str(n) for n in BD["names"]] if BD is not None else []
PT_NAMES = set(str(n) for n in PT["names"]) if PT is not None else set()

Z_MAX = 4.5
XMED_MAX = 1.5
# the subset rendered without t = 1 connections (use_t1_paths = false)
NO_T1 = [n for n in NAMES if n + "/nt0" in BD] if BD is not None else []


def _agrees_with_pt(name):
    """The reference's bidirectional and path-traced fixtures agree, with a
    margin (channel means within 2.5 standard errors: the GPU's halves have
    twice the samples, so a bias the fixtures' noise hides shows there), and
    the scene has no Phong surface (on those the reference's bidirectional
    tracer is darker by 0.1-2 %, a bias the GPU reproduces)."""
    if "_glos_" in name or "phong" in name:
        return False
    r = ptcheck.compare_blocks(BD[name + "/rb0"], BD[name + "/rb1"], PT[name + "/rb0"],
                               PT[name + "/rb1"])
    return bool(np.all(np.abs(r["mean_z"]) < 2.5) and r["Xmed"] < XMED_MAX)


AGREE = ([n for n in NAMES if n in PT_NAMES and _agrees_with_pt(n)]
         if BD is not None and PT is not None else [])


def _render(name, spp, seeds=(101, 102), use_t1=True):
    import dort_b200 as db
    case = ref_scenes.case_by_name(name)
    d = ref_scenes.build(case)
    sc = db.scene_from_dict(d)
    out = []
    for seed in seeds:
        p = db.render_params(d["camera"], case["width"], case["height"], spp,
                             min_depth=case["min_depth"], max_depth=case["max_depth"],
                             seed=seed, renderer="bdpt", use_t1_paths=use_t1)
        img, st = sc.render(p)
        assert st["samples"] + st["dropped"] == case["width"] * case["height"] * spp
        assert st["dropped"] <= 1e-4 * st["samples"]
        out.append(ptcheck.block_means(img.astype(np.float64)))
    sc.close()
    return out


def _assert_close(name, ours, ref0, ref1):
    r = ptcheck.compare_blocks(ours[0], ours[1], ref0, ref1)
    ref_mean = (np.asarray(ref0, np.float64) + np.asarray(ref1, np.float64)).mean(axis=(0, 1)) / 2
    lit = ref_mean > 1e-4
    ours_mean = (np.asarray(ours[0]) + np.asarray(ours[1])).mean(axis=(0, 1)) / 2
    assert np.all(ours_mean[~lit] < 1e-4), (name, ours_mean, ref_mean)
    if lit.any():
        assert np.all(np.abs(r["mean_z"][lit]) < Z_MAX), (name, r)
        assert r["Xmed"] < XMED_MAX, (name, r)


@pytest.mark.gpu
@pytest.mark.skipif(BD is None, reason="tests/golden/bdpt_images.npz missing")
@pytest.mark.parametrize("name", NAMES)
def test_bdpt_matches_reference_bdpt(name, cuda):
    ours = _render(name, int(BD["spp"]))
    _assert_close(name, ours, BD[name + "/rb0"], BD[name + "/rb1"])


@pytest.mark.gpu
@pytest.mark.skipif(BD is None, reason="tests/golden/bdpt_images.npz missing")
@pytest.mark.parametrize("name", NO_T1)
def test_bdpt_without_t1_paths_matches_reference_bdpt(name, cuda):
    ours = _render(name, int(BD["spp"]), seeds=(301, 302), use_t1=False)
    _assert_close(name, ours, BD[name + "/nt0"], BD[name + "/nt1"])


@pytest.mark.gpu
@pytest.mark.skipif(BD is None or PT is None, reason="fixtures missing")
@pytest.mark.parametrize("name", AGREE)
def test_bdpt_converges_to_the_path_tracer(name, cuda):
    ours = _render(name, 2 * int(BD["spp"]), seeds=(201, 202))
    _assert_close(name, ours, PT[name + "/rb0"], PT[name + "/rb1"])


@pytest.mark.gpu
def test_bdpt_entry_points(cuda):
    import dort_b200 as db
    case = ref_scenes.case_by_name("box_diff_area_pin")
    d = ref_scenes.build(case)
    sc = db.scene_from_dict(d)
    p = db.render_params(d["camera"], 64, 64, 2, max_depth=3, renderer="bdpt")
    img, st = sc.render(p)
    assert img.shape == (64, 64, 3) and np.isfinite(img).all() and img.mean() > 0
    assert st["rays"] > 0 and st["samples"] == 64 * 64 * 2
    with pytest.raises(db.DortError, match="DORT_ERR_UNSUPPORTED"):
        sc.render_wavefront(p)
    with pytest.raises(db.DortError, match="max_depth"):
        sc.render(db.render_params(d["camera"], 64, 64, 1, max_depth=14, renderer="bdpt"))
    sc.close()


HOST_CASES = ["box_diff_area_pin", "box_glos_sphe_pin", "box_delt_dire_pin", "box_diff_poin_pin",
              "openbox_glos_infi_pin", "box_diff_area_orth_d2", "box_diff_area_thin_d1",
              "simple_sphe_glos_area_fwd_pin", "simple_disk_diff_mixd_2_pin",
              "bsdf_dielectric_1.5@square", "bsdf_phong_50@square"]


def _device_and_host(case, d, w, h, spp, use_t1, max_depth=None, seed=17):
    import dort_b200 as db
    p = db.render_params(d["camera"], w, h, spp, min_depth=case["min_depth"],
                         max_depth=case["max_depth"] if max_depth is None else max_depth,
                         seed=seed, renderer="bdpt", use_t1_paths=use_t1)
    sc = db.scene_from_dict(d)
    dev, st = sc.render(p)
    sc.close()
    return dev, db.host_check_render(d, p), st


@pytest.mark.gpu
@pytest.mark.parametrize("name", HOST_CASES)
@pytest.mark.parametrize("use_t1", [True, False])
def test_bdpt_device_equals_host_check(name, use_t1, cuda):
    """The device's connection-parallel kernels (walks, one launch per
    connection case, the ordered per-sample gather) against the same
    estimator run one sample at a time by the host check, on the same random
    numbers: the same image up to float rounding (the film's atomic sums,
    fused multiply-adds) and at most a few paths that take another branch
    at an edge or a critical angle."""
    case = ref_scenes.case_by_name(name)
    d = ref_scenes.build(case)
    dev, host, st = _device_and_host(case, d, 24, 20, 16, use_t1)
    assert st["samples"] + st["dropped"] == 24 * 20 * 16
    assert host.mean() > 0
    assert ptcheck.forked_pixels(dev, host, tol=1e-3) <= 3, name
    assert abs(dev.mean() / host.mean() - 1) < 2e-3, name


@pytest.mark.gpu
def test_bdpt_device_equals_host_check_at_depth_13(cuda):
    """max_depth 13, the deepest the tracer takes: 15 vertices per walk and
    120 connection slots per sample (all four words of the gather's mask)."""
    case = ref_scenes.case_by_name("box_diff_area_pin")
    d = ref_scenes.build(case)
    dev, host, _ = _device_and_host(case, d, 16, 16, 16, True, max_depth=13)
    assert ptcheck.forked_pixels(dev, host, tol=1e-3) <= 3
    assert abs(dev.mean() / host.mean() - 1) < 2e-3


@pytest.mark.gpu
@pytest.mark.parametrize("min_depth,max_depth", [(2, 6), (4, 4), (1, 1)])
def test_bdpt_device_equals_host_check_depth_window(min_depth, max_depth, cuda):
    """Connections outside [min_depth + 2, max_depth + 2] vertices are
    neither listed nor given a slot (a window of one length, and max_depth
    1: no s, t >= 2 connection at all)."""
    import dort_b200 as db
    case = ref_scenes.case_by_name("box_glos_sphe_pin")
    d = ref_scenes.build(case)
    p = db.render_params(d["camera"], 20, 16, 16, min_depth=min_depth, max_depth=max_depth,
                         seed=29, renderer="bdpt")
    sc = db.scene_from_dict(d)
    dev, _ = sc.render(p)
    sc.close()
    host = db.host_check_render(d, p)
    assert host.mean() > 0
    assert ptcheck.forked_pixels(dev, host, tol=1e-3) <= 3
    assert abs(dev.mean() / host.mean() - 1) < 2e-3


@pytest.mark.gpu
def test_bdpt_frame_spanning_two_chunks(cuda):
    """32 x 32 x 1100 samples: more than one chunk of 2^20 samples, so the
    walk buffers, lists and slots are reused by the second chunk."""
    case = ref_scenes.case_by_name("box_diff_area_pin")
    d = ref_scenes.build(case)
    dev, host, st = _device_and_host(case, d, 32, 32, 1100, True)
    assert st["samples"] + st["dropped"] == 32 * 32 * 1100
    assert ptcheck.forked_pixels(dev, host, tol=1e-3) <= 3
    assert abs(dev.mean() / host.mean() - 1) < 1e-3


@pytest.mark.gpu
def test_bdpt_scene_without_lights_keeps_black_samples(cuda):
    """No light: every sample is 0 and kept (sample_path returns at once),
    and no connection is listed."""
    import dort_b200 as db
    from dort_b200 import scenes
    sd = scenes.cornell_box()
    sd["tri_emission"] = np.zeros_like(sd["tri_emission"])
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 40, 30, 4, max_depth=8, renderer="bdpt")
    img, st = sc.render(p)
    sc.close()
    assert st["samples"] == 40 * 30 * 4 and st["dropped"] == 0
    assert not img.any()


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,spp", [(1, 1, 3), (3, 1, 349526), (7, 5, 1)])
def test_bdpt_small_and_ragged_sample_counts(w, h, spp, cuda):
    """Partial warps and blocks: a single pixel with 3 samples, a frame whose
    second chunk holds two samples (3 x 349,526 = 2^20 + 2), an odd 7 x 5
    frame."""
    import dort_b200 as db
    from dort_b200 import scenes
    sd = scenes.cornell_box()
    p = db.render_params(sd["camera"], w, h, spp, max_depth=5, seed=13, renderer="bdpt")
    sc = db.scene_from_dict(sd)
    dev, st = sc.render(p)
    sc.close()
    assert st["samples"] + st["dropped"] == w * h * spp
    host = db.host_check_render(sd, p)
    assert np.isfinite(dev).all()
    if spp > 1000:
        assert abs(dev.mean() / host.mean() - 1) < 1e-3
    else:
        assert ptcheck.forked_pixels(dev, host, tol=1e-3) == 0


def test_bdpt_fixture_is_consistent():
    """CPU: the fixture covers the reference's "bdpt" test scenes with the
    expected shapes."""
    if BD is None:
        pytest.skip("fixture missing")
    assert len(NAMES) >= 70 and len(NO_T1) >= 5 and len(AGREE) >= 30
    for name in NAMES:
        case = ref_scenes.case_by_name(name)
        by, bx = (case["height"] + 15) // 16, (case["width"] + 15) // 16
        assert BD[name + "/rb0"].shape == (by, bx, 3)
        assert BD[name + "/rb1"].shape == (by, bx, 3)


def test_bdpt_statistics_flag_a_planted_bias():
    """CPU: the reference's halves against the same halves scaled by 5 % (a
    mistake planted on the reference side) fail the checks on at least 90 %
    of the lit fixture scenes."""
    if BD is None:
        pytest.skip("fixture missing")
    flagged = lit_scenes = 0
    for name in NAMES:
        b0 = np.asarray(BD[name + "/rb0"], np.float64)
        b1 = np.asarray(BD[name + "/rb1"], np.float64)
        lit = (b0 + b1).mean(axis=(0, 1)) > 1e-4
        if not lit.any():
            continue
        lit_scenes += 1
        bad = ptcheck.compare_blocks(b0 * 1.05, b1 * 1.05, b0, b1)
        flagged += bool(np.any(np.abs(bad["mean_z"][lit]) >= Z_MAX) or bad["Xmed"] >= XMED_MAX)
    assert lit_scenes >= 60 and flagged >= 0.9 * lit_scenes
