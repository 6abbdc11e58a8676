"""Generates the converged reference images in tests/golden/pt_golden.npz.

Every image is rendered by the reference renderer's own "pt" PathRenderer
(src/dort/path_renderer.cpp) compiled from its sources into
oracle/_ref/libdort_ref.so and driven by oracle/ref/pt_harness.cpp, which
assembles the scene the way the reference's Lua builder does.  Each image is
two independent halves (different sampler seeds), stored separately, so tests
can estimate the reference's own Monte Carlo noise.

The reference's thread pool crashes intermittently with more than one
worker (a race in its thread_pool.cpp), so the halves are rendered by
single-threaded reference processes in parallel and averaged.

    make -C oracle ref REF=<reference tree> && python tests/golden/gen_images.py
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "pt_golden.npz")

# name -> (scene factory, width, height, spp per half, render kwargs)
CASES = {
    "cornell_c1": ("cornell", {}, 64, 64, 2048, {"max_depth": 8}),
    "cornell_glos": ("variant", {"kind": "glos"}, 48, 48, 1024, {"max_depth": 5}),
    "cornell_delt": ("variant", {"kind": "delt"}, 48, 48, 1024, {"max_depth": 5}),
    "cornell_infi": ("variant", {"kind": "diff", "light": "infi"}, 48, 48, 512,
                     {"max_depth": 5}),
    "env_boxes": ("env", {}, 48, 48, 512, {"max_depth": 6}),
}


def make_scene(kind, kw):
    from dort_b200 import scenes
    if kind == "cornell":
        return scenes.cornell_box()
    if kind == "variant":
        return scenes.cornell_variant(**kw)
    return scenes.env_test_scene(**kw)


def _job(args):
    name, seed, spp = args
    from oracle import pyoracle as po
    kind, kw, w, h, _, rkw = CASES[name]
    sc = make_scene(kind, kw)
    img, secs = po.ref_pt_render(sc, w, h, spp, seed=seed, threads=1, **rkw)
    return name, seed, img, secs


def main():
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    chunks = 8                        # per half
    jobs = []
    for name, (_, _, _, _, spp, _) in CASES.items():
        for half in range(2):
            for c in range(chunks):
                jobs.append((name, 1000 * (half + 1) + c, spp // chunks))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        results = pool.map(_job, jobs)
    arrays = {}
    for name in CASES:
        for half in range(2):
            imgs = [img for (n, seed, img, _) in results
                    if n == name and seed // 1000 == half + 1]
            arrays[f"{name}_half{half}"] = np.mean(imgs, axis=0).astype(np.float32)
        spp = CASES[name][4]
        arrays[f"{name}_spp_per_half"] = np.array(spp, np.int64)
        print(name, arrays[f"{name}_half0"].mean(axis=(0, 1)), arrays[f"{name}_half1"].mean(axis=(0, 1)))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
