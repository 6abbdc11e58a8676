"""Path-tracer parity on the GPU.

* Against the reference: the committed golden images were rendered by the
  reference's own PathRenderer (tests/golden/gen_images.py).  Renders are
  Monte Carlo estimates with different random streams, so the bar is
  statistical: the block-chi-square ratio X of tests/ptcheck.py stays below
  3.5 (about 1 when both sides estimate the same image) and every channel
  mean agrees within 2 %.
* Between this build's renderers: the megakernel, the wavefront renderer and
  the host-compiled path sampler draw the same random numbers per pixel and
  sample, so their images agree to float rounding.
"""
import os
import sys

import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from tests import ptcheck

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, "golden"))
import gen_images as gi  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "pt_golden.npz"))


@pytest.mark.parametrize("name", list(gi.CASES))
@pytest.mark.parametrize("renderer", ["mega", "wavefront"])
def test_matches_reference_golden(cuda, name, renderer):
    kind, kw, w, h, spp, rkw = gi.CASES[name]
    sd = gi.make_scene(kind, kw)
    sc = db.scene_from_dict(sd)
    halves = []
    for seed in (11, 12):
        p = db.render_params(sd["camera"], w, h, spp * 4, seed=seed, **rkw)
        img = sc.render(p)[0] if renderer == "mega" else sc.render_wavefront(p)[0]
        halves.append(img)
    r = ptcheck.compare(halves[0], halves[1], GOLDEN[f"{name}_half0"], GOLDEN[f"{name}_half1"])
    assert np.all(r["X"] < 3.5), r
    assert np.all(np.abs(r["mean_rel"]) < 0.02), r


@pytest.mark.parametrize("name", ["cornell_c1", "cornell_delt", "env_boxes"])
def test_wavefront_equals_megakernel(cuda, name):
    kind, kw, w, h, spp, rkw = gi.CASES[name]
    sd = gi.make_scene(kind, kw)
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], w, h, 64, seed=3, **rkw)
    a, sa = sc.render(p)
    b, sb = sc.render_wavefront(p)
    assert ptcheck.rel_rmse(b, a) < 2e-3
    assert abs(sa["rays"] - sb["rays"]) <= 0.001 * sa["rays"]


def test_megakernel_matches_host_compiled_sampler(cuda):
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 24, 16, 8, max_depth=8, seed=9)
    g, _ = sc.render(p)
    hcpu = db.host_check_render(sd, p)
    assert ptcheck.rel_rmse(g, hcpu) < 1e-4


def test_render_is_deterministic(cuda):
    sd = scenes.cornell_variant("glos")
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 40, 30, 16, seed=5)
    a, _ = sc.render(p)
    b, _ = sc.render(p)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


C1_FULL = np.load(os.path.join(HERE, "golden", "c1_full.npz"))


def test_cornell_config_full_size(cuda):
    """The CPU-runnable benchmark configuration, 256x256, 64 spp, depth 8,
    against the reference PathRenderer's render of it at that size
    (tests/golden/gen_c1_full.py: two halves of 256 spp as 4x4 block means):
    two GPU halves at the configuration's 64 spp, per block."""
    import gen_c1_full as g1
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    halves = []
    for seed in (42, 43):
        p = db.render_params(sd["camera"], 256, 256, 64, max_depth=8, seed=seed)
        img, st = sc.render(p)
        assert st["samples"] == 256 * 256 * 64 and st["dropped"] == 0
        assert st["rays"] > st["samples"]
        halves.append(g1.block_means(img))
    r = ptcheck.compare_blocks(halves[0], halves[1], C1_FULL["half0"], C1_FULL["half1"])
    assert np.all(np.abs(r["mean_z"]) < 4.5), r
    assert r["Xmed"] < 1.5, r
    wimg, wst = sc.render_wavefront(p)
    assert ptcheck.rel_rmse(wimg, img) < 2e-3


@pytest.mark.parametrize("variant", ["cornell", "delt", "infi"])
def test_wavefront_sample_all_lights_equals_megakernel(cuda, variant):
    """Every light sampled at every vertex (sample_all_lights): the wavefront
    queues one set of direct-lighting rays per light and path and traces the
    megakernel's paths (same random numbers)."""
    sd = {"cornell": lambda: scenes.cornell_box(),
          "delt": lambda: scenes.cornell_variant("delt"),
          "infi": lambda: scenes.cornell_variant("diff", light="both")}[variant]()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 48, 32, 16, max_depth=6, sample_all_lights=True, seed=8)
    a, sa = sc.render(p)
    b, sb = sc.render_wavefront(p)
    assert a.mean() > 0
    # the same paths: at most a pixel or two whose path forks at a float
    # rounding difference between the two kernels
    assert ptcheck.forked_pixels(b, a) <= 2
    assert abs(sa["rays"] - sb["rays"]) <= 0.001 * sa["rays"]
    # and in a batch, beside a job that picks one light: the batch's frames
    # equal the wavefront's single frames
    p1 = db.render_params(sd["camera"], 40, 24, 8, max_depth=6, seed=9)
    bt = db.Batch([(sc, p), (sc, p1)])
    bt.render()
    assert ptcheck.forked_pixels(bt.image(0), b) == 0
    assert ptcheck.forked_pixels(bt.image(1), sc.render_wavefront(p1)[0]) == 0
    assert ptcheck.forked_pixels(bt.image(1), sc.render(p1)[0]) <= 2
    bt.close()


@pytest.mark.parametrize("sort_rays,staged", [(False, False), (True, False), (False, True)])
@pytest.mark.parametrize("capacity,block", [(64, 32), (4096, 256), (100000, 128), (50000, 512)])
def test_wavefront_queue_shapes(cuda, capacity, block, sort_rays, staged):
    """Queue sizes, block sizes, the optional ray sort and the staging of the
    shadow queue through bulk copies (blocks above 256 threads load it
    directly) change the order of work, not the paths: the same image as the
    megakernel."""
    sd = scenes.cornell_variant("delt")
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 32, 24, 16, seed=4)
    a, _ = sc.render(p)
    b, st = sc.render_wavefront(p, {"queue_capacity": capacity, "trace_block": block,
                                    "shade_block": block, "sort_rays": sort_rays,
                                    "stage_queues": staged})
    assert ptcheck.rel_rmse(b, a) < 2e-3
    assert st["waves"] >= 1


def test_wavefront_deterministic_sums(cuda):
    """With deterministic sums (per-unit sums added in unit order) the same
    frame renders to the same bits, the megakernel's image up to rounding;
    batches refuse the option."""
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 40, 32, 23, max_depth=5, seed=21)
    a, _ = sc.render_wavefront(p, {"deterministic": True})
    b, _ = sc.render_wavefront(p, {"deterministic": True, "queue_capacity": 1024})
    c, _ = sc.render_wavefront(p, {"deterministic": True})
    assert np.array_equal(a, c) and np.array_equal(a, b)
    m, _ = sc.render(p)
    assert ptcheck.forked_pixels(a, m) <= 2
    # and the atomic film again afterwards
    d, _ = sc.render_wavefront(p)
    assert ptcheck.forked_pixels(d, m) <= 2
    with pytest.raises(db.DortError) as e:
        db.Batch([(sc, p)], {"deterministic": True})
    assert e.value.status == -5
