"""Generates tests/golden/c1_full.npz: the Cornell box of the CPU benchmark
configuration (256 x 256, depth 8) rendered by the reference renderer's own
"pt" PathRenderer (compiled from its sources into oracle/_ref), as two
independent halves of SPP samples per pixel stored as 4 x 4 pixel block means.

The reference's thread pool crashes intermittently with more than one
worker, so the halves are split into chunks rendered by single-threaded
reference processes in parallel and averaged.

    make -C oracle ref && python tests/golden/gen_c1_full.py
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "c1_full.npz")
W, H, DEPTH, SPP, BLOCK = 256, 256, 8, 256, 4
CHUNKS = 8                     # per half


def _job(seed):
    from dort_b200 import scenes
    from oracle import pyoracle as po
    img, secs = po.ref_pt_render(scenes.cornell_box(), W, H, SPP // CHUNKS, max_depth=DEPTH,
                                 seed=seed, threads=1)
    return seed, img, secs


def block_means(img, b=BLOCK):
    h, w = img.shape[0] // b * b, img.shape[1] // b * b
    return img[:h, :w].astype(np.float64).reshape(h // b, b, w // b, b, 3).mean(axis=(1, 3))


def main():
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    seeds = [1000 * (half + 1) + c for half in range(2) for c in range(CHUNKS)]
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs) as pool:
        results = pool.map(_job, seeds)
    out = {}
    for half in range(2):
        imgs = [img for (seed, img, _) in results if seed // 1000 == half + 1]
        out[f"half{half}"] = block_means(np.mean(imgs, axis=0)).astype(np.float32)
    out["spp_per_half"] = np.int32(SPP)
    out["size"] = np.array([W, H, DEPTH, BLOCK], np.int32)
    np.savez_compressed(OUT, **out)
    print(f"{time.time() - t0:.0f}s; means {out['half0'].mean(axis=(0, 1))} "
          f"{out['half1'].mean(axis=(0, 1))} -> {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
