"""Fixture tests/golden/lt_images.npz for the light tracer's parity.

The reference's image tests render the "lt" renderer (LightRenderer,
src/dort/light_renderer.cpp) on its Cornell boxes with diffuse surfaces
(test_box.lua:200-226), on the simple scenes with non-mirror surfaces
(test_simple.lua:186-196) and on every material sphere (test_bsdf.lua:
108-150).  The material-sphere images are 512 x 338, and on films wider than
high the reference's light tracer crashes (Film::add_splat sizes a
variable-length array from an empty pixel rectangle for the film positions
outside the film that PinholeCamera::get_film_pos returns, film.cpp:32-41,
pinhole_camera.cpp:107-122; reproduced here), so they are rendered square
here ("<name>@square", ref_scenes.case_by_name).  For the cases listed in
LT_CASES this stores the same scene rendered by the
reference's current "lt" code (compiled from its sources into
oracle/_ref/libdort_ref.so, oracle/ref/scene_harness.cpp) at SPP iterations:

    <name>/rb   16x16 block means

One render per scene: LightRenderer seeds each of its jobs with the job's
index alone (sampler->split(job_i), light_renderer.cpp:29-31, and
RandomSampler::split starts a new generator from that seed,
random_sampler.cpp:31-33), so its image does not depend on the render's seed
and two "halves" would be the same image.  The tests take its noise from the
GPU's independent halves, scaled by the ratio of sample counts.

    make -C oracle ref && python tests/golden/gen_lt_images.py
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

SPP = int(os.environ.get("LT_IMAGES_SPP", "128"))
OUT = os.path.join(HERE, "lt_images.npz")

LT_CASES = (
    ["box_diff_area_pin", "box_diff_poin_pin", "box_diff_dire_pin", "box_diff_area_thin"] +
    [f"simple_{g}_{s}_{l}_pin" for g in ("sphe", "disk", "cube", "disk2")
     for s in ("diff", "glos") for l in ("poin_fwd", "area_fwd", "dire_blw", "mixd_2")] +
    [f"bsdf_{m}@square" for m in ("lamb", "orennayar_0.1", "mirror", "dielectric_1.5",
                                  "dielectric_inv1.5", "phong_10", "phong_200")])


def _job(args):
    name, seed = args
    import dort_b200 as db
    import pyoracle
    import ptcheck
    import ref_scenes
    case = ref_scenes.case_by_name(name)
    sc = ref_scenes.build(case)
    p = db.render_params(sc["camera"], case["width"], case["height"], SPP,
                         min_depth=case["min_depth"], max_depth=case["max_depth"], seed=seed,
                         renderer="lt")
    img, secs = pyoracle.ref_scene_render(sc, p)
    return name, seed, ptcheck.block_means(img).astype(np.float32), secs


def main() -> None:
    import ref_scenes
    for n in LT_CASES:
        ref_scenes.case_by_name(n)
    jobs = [(n, 1) for n in LT_CASES]
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    out = {}
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs) as pool:
        for name, seed, blocks, secs in pool.imap_unordered(_job, jobs):
            out[f"{name}/rb"] = blocks
            print(f"{name:40s} {secs:6.1f}s  ({time.time() - t0:.0f}s)", flush=True)
    out["names"] = np.asarray(LT_CASES)
    out["spp"] = np.int32(SPP)
    np.savez_compressed(OUT, **out)
    print(f"{len(LT_CASES)} cases -> {OUT}")


if __name__ == "__main__":
    main()
