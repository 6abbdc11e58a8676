"""Fixture tests/golden/bdpt_images.npz for the bidirectional tracer's parity.

The reference's image tests render the "bdpt" renderer (BdptRenderer,
src/dort/bdpt_renderer.cpp) on its Cornell boxes (test_box.lua:199-223, the
cases with an image here: no environment-map scenes), on every simple scene
(test_simple.lua:141-222) and on every material sphere (test_bsdf.lua:
100-150).  The material-sphere images are 512 x 338; the bidirectional
tracer's t = 1 connections splat through Film::add_splat like the light
tracer, which crashes on films wider than high (film.cpp:32-41 sizes an
array from an empty pixel rectangle for positions outside the film), so
they are rendered square here ("<name>@square", ref_scenes.case_by_name).
For every case of BDPT_CASES this stores the scene rendered by the
reference's current "bdpt" code (compiled from its sources into
oracle/_ref/libdort_ref.so, oracle/ref/scene_harness.cpp) as two
independent halves (seeds 1 and 2: its tiles are seeded from the render's
sampler, renderer.cpp:55-75) of SPP iterations:

    <name>/rb0, <name>/rb1   16x16 block means of the halves
    <name>/nt0, <name>/nt1   the same without t = 1 connections
                             (use_t1_paths = false; NO_T1 cases only)

    make -C oracle ref && python tests/golden/gen_bdpt_images.py
"""
from __future__ import annotations

import multiprocessing as mp
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

SPP = int(os.environ.get("BDPT_IMAGES_SPP", "32"))
OUT = os.path.join(HERE, "bdpt_images.npz")
# rendered a second time without t = 1 connections
NO_T1 = ["box_diff_area_pin", "box_glos_sphe_pin", "box_delt_dire_pin",
         "simple_sphe_glos_area_fwd_pin", "bsdf_dielectric_1.5@square"]


def _cases():
    import ref_scenes
    box = [c["name"] for c in ref_scenes.CASES
           if c["name"].split("_")[0] in ("box", "openbox") and not re.search(r"_d\d$", c["name"])
           and not c["name"].startswith(("box_delt_area", "box_delt_poin"))]
    simple = [c["name"] for c in ref_scenes.CASES if c["name"].startswith("simple_")]
    bsdf = [c["name"] + "@square" for c in ref_scenes.CASES if c["name"].startswith("bsdf_")]
    return box + simple + bsdf


def _job(args):
    name, seed, use_t1 = args
    import dort_b200 as db
    import pyoracle
    import ptcheck
    import ref_scenes
    case = ref_scenes.case_by_name(name)
    sc = ref_scenes.build(case)
    p = db.render_params(sc["camera"], case["width"], case["height"], SPP,
                         min_depth=case["min_depth"], max_depth=case["max_depth"], seed=seed,
                         renderer="bdpt", use_t1_paths=use_t1)
    img, secs = pyoracle.ref_scene_render(sc, p)
    return name, seed, use_t1, ptcheck.block_means(img).astype(np.float32), secs


def main() -> None:
    names = _cases()
    only = os.environ.get("BDPT_IMAGES_ONLY_NO_T1") == "1"
    jobs = [] if only else [(n, s, True) for n in names for s in (1, 2)]
    jobs += [(n, s, False) for n in NO_T1 for s in (3, 4)]
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    # BDPT_IMAGES_ONLY_NO_T1=1 adds the use_t1_paths = false renders to an
    # existing fixture
    out = dict(np.load(OUT)) if only else {}
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs) as pool:
        for name, seed, use_t1, blocks, secs in pool.imap_unordered(_job, jobs):
            out[f"{name}/{'rb' if use_t1 else 'nt'}{(seed - 1) % 2}"] = blocks
            print(f"{name:40s} {seed} {secs:6.1f}s  ({time.time() - t0:.0f}s)", flush=True)
    out["names"] = np.asarray(names)
    out["spp"] = np.int32(SPP)
    np.savez_compressed(OUT, **out)
    print(f"{len(names)} cases -> {OUT}")


if __name__ == "__main__":
    main()
