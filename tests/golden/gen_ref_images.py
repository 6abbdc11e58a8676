"""Fixture tests/golden/ref_images.npz for the reference test-scene parity.

For every case of ref_scenes.CASES whose image exists in the reference tree
(test/ref/<name>.hdr, the reference's stored converged image of that test
scene), two things are stored:

1. The stored image, reduced to what the reference's own image test reads
   (test_convergence, src/dort/convergence_test.cpp:10-101, min tile 32):
     <name>/tiles    x0, y0, x1, y1 of every tile it checks
     <name>/tmeans   the stored image's mean RGB over each tile
     <name>/blocks   the stored image's mean RGB over 16x16 blocks
   read as the reference's tests read it (RGBE, value = m * 2^(e - 136)).

2. The same scene rendered here by the reference's *current* code (its
   PathRenderer and scene classes compiled from its sources into
   oracle/_ref/libdort_ref.so, assembled by oracle/ref/scene_harness.cpp),
   as two independent halves (seeds 1 and 2) of SPP samples per pixel:
     <name>/rb0, <name>/rb1   16x16 block means of the halves
     <name>/conv              test_convergence's worst tile ratio of that
                              render against the stored image (<= 1: the
                              reference's own test passes; > 1: the stored
                              image no longer matches the reference's code)

The halves are rendered by single-threaded reference processes in parallel
(the reference's thread pool is not safe with several workers).

    make -C oracle ref && python tests/golden/gen_ref_images.py [reference tree]
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

SPP = int(os.environ.get("REF_IMAGES_SPP", "32"))
OUT = os.path.join(HERE, "ref_images.npz")


def _job(args):
    name, seed = args
    import dort_b200 as db
    import pyoracle
    import ptcheck
    import ref_scenes
    case = next(c for c in ref_scenes.CASES if c["name"] == name)
    sc = ref_scenes.build(case)
    p = db.render_params(sc["camera"], case["width"], case["height"], SPP,
                         min_depth=case["min_depth"], max_depth=case["max_depth"],
                         sample_all_lights=case["sample_all_lights"], seed=seed)
    img, secs = pyoracle.ref_scene_render(sc, p)
    return name, seed, img, ptcheck.block_means(img).astype(np.float32), secs


def main(ref_root: str) -> None:
    import ptcheck
    import ref_scenes
    from dort_b200.image import read_rgbe
    out, names, golden = {}, [], {}
    for case in ref_scenes.CASES:
        path = os.path.join(ref_root, "test", "ref", case["name"] + ".hdr")
        if not os.path.exists(path):
            continue
        img = read_rgbe(path).astype(np.float64)
        assert img.shape == (case["height"], case["width"], 3), (case["name"], img.shape)
        tiles = ptcheck.convergence_tiles(case["width"], case["height"])
        n = case["name"]
        out[n + "/tiles"] = tiles
        out[n + "/tmeans"] = ptcheck.tile_means(img, tiles).astype(np.float32)
        out[n + "/blocks"] = ptcheck.block_means(img).astype(np.float32)
        golden[n] = case
        names.append(n)

    jobs = [(n, seed) for n in names for seed in (1, 2)]
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    t0 = time.time()
    halves = {}
    with mp.get_context("spawn").Pool(procs) as pool:
        for name, seed, img, blocks, secs in pool.imap_unordered(_job, jobs):
            out[f"{name}/rb{seed - 1}"] = blocks
            halves.setdefault(name, {})[seed] = img
            if len(halves[name]) == 2:
                full = (halves[name][1] + halves[name][2]) / 2
                case = golden[name]
                worst, _ = ptcheck.reference_convergence(
                    out[name + "/tmeans"], out[name + "/tiles"], full,
                    variation=case["variation"])
                out[name + "/conv"] = np.float32(worst)
                del halves[name]
                print(f"{name:40s} conv {worst:6.2f}  ({time.time() - t0:.0f}s)", flush=True)
    out["names"] = np.asarray(names)
    out["spp"] = np.int32(SPP)
    np.savez_compressed(OUT, **out)
    print(f"{len(names)} cases -> {OUT}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else
         os.environ.get("DORT_REFERENCE_TREE") or os.path.join(os.path.dirname(ROOT), "reference"))
