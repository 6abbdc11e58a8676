"""Generates tests/golden/c3_images.npz: the 1080p benchmark scene rendered by
the reference renderer's own "pt" PathRenderer at a reduced resolution.

The scene is dort_b200.scenes.wavefront_scene() -- the 1,997,122-triangle
fBm-displaced icosphere and ground plane under the procedural 1024 x 512 HDR
sky, camera and depth 16 of the benchmark -- with every GGX conductor patch
given a Lambert material of the conductor's colour instead (the reference has
no GGX conductor).  It is rendered at 240 x 135 (the benchmark camera, 1/8 of
the resolution per axis) by the reference's PathRenderer compiled from its
sources into oracle/_ref (oracle/ref/pt_harness.cpp builds the scene the way
its Lua builder does), as two independent halves of SPP samples per pixel.
The halves are stored as 4 x 4 pixel block means (tests compare block means).

The reference's thread pool crashes intermittently with more than one worker,
so the halves are split into chunks rendered by single-threaded reference
processes in parallel and averaged.

    make -C oracle ref && python tests/golden/gen_c3_images.py
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

OUT = os.path.join(HERE, "c3_images.npz")
W, H, DEPTH, SPP, BLOCK = 240, 135, 16, 1024, 4
CHUNKS = 16                    # per half


def c3_parity_scene():
    """The benchmark scene with its conductors turned Lambert (same patches,
    same colours)."""
    from dort_b200 import scenes
    sd = scenes.wavefront_scene()
    sd["materials"] = [({"kind": 0, "color": m["color"]} if m.get("kind") == 4 else m)
                       for m in sd["materials"]]
    return sd


_scene = None


def _init():
    global _scene
    from oracle import pyoracle as po
    _scene = po.RefPtScene(c3_parity_scene(), threads=1)


def _job(seed):
    img, secs = _scene.render(W, H, SPP // CHUNKS, max_depth=DEPTH, seed=seed, threads=1)
    return seed, img, secs


def block_means(img, b=BLOCK):
    h, w = img.shape[0] // b * b, img.shape[1] // b * b
    return img[:h, :w].astype(np.float64).reshape(h // b, b, w // b, b, 3).mean(axis=(1, 3))


def main():
    procs = int(os.environ.get("GOLDEN_PROCS", str(os.cpu_count() or 1)))
    seeds = [1000 * (half + 1) + c for half in range(2) for c in range(CHUNKS)]
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs, initializer=_init) as pool:
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
