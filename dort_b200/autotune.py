"""Autotuner for the wavefront renderer.

Picks the wavefront's queue capacity (paths in flight), the thread-block
sizes of its trace and shade stages and the BVH node width by timing short
proxy frames of the caller's own scene and camera on the GPU: the same
resolution and depth at a few samples per pixel, each candidate run twice
with the faster run kept (the first warms caches).  The proxy keeps every
sample the full frame would trace at sample 0..k, so the ranking reflects the
real frame's ray mix.

    best = autotune(scene_dict, params)          # -> {"bvh_width": 8, "tuning": {...}}
    sc = Scene(..., bvh_width=best["bvh_width"])
    sc.render_wavefront(params, best["tuning"])
"""
from __future__ import annotations

import copy
import itertools
import time

from . import _abi, render_params, scene_from_dict

# more path slots make fewer, fuller waves (the 1080p frame at 256 spp:
# 567 / 606 M samples/s at 2^22 / 2^24); about 330 B of device memory each
DEFAULT_CAPACITIES = (1 << 22, 1 << 23, 1 << 24)
DEFAULT_BLOCKS = (64, 128, 256)
DEFAULT_WIDTHS = (8, 4)


def _time_frame(sc, params, tuning) -> float:
    best = float("inf")
    for _ in range(2):
        _, st = sc.render_wavefront(params, tuning)
        best = min(best, st["ms"])
    return best


def autotune(scene: dict, params: _abi.RenderParams, proxy_spp: int = 4,
             capacities=DEFAULT_CAPACITIES, blocks=DEFAULT_BLOCKS, widths=DEFAULT_WIDTHS,
             budget_s: float = 60.0, log=None) -> dict:
    """Returns {"bvh_width", "tuning", "ms", "table"}: the fastest candidate
    on a proxy frame of `proxy_spp` samples per pixel."""
    proxy = copy.copy(params)
    proxy = render_params(scene["camera"], params.width, params.height,
                          min(params.iterations, proxy_spp), min_depth=params.min_depth,
                          max_depth=params.max_depth, only_direct=bool(params.only_direct),
                          direct_strategy={0: "mis", 1: "bsdf", 2: "light"}[params.direct_strategy],
                          seed=params.seed)
    samples = params.width * params.height * proxy.iterations
    table = []
    t0 = time.perf_counter()
    best = None
    for width in widths:
        sc = scene_from_dict(scene, bvh_width=width)
        for cap, tb, sb in itertools.product(capacities, blocks, blocks):
            if cap > 4 * samples and cap != min(capacities):
                continue
            if time.perf_counter() - t0 > budget_s:
                break
            tuning = {"queue_capacity": cap, "trace_block": tb, "shade_block": sb}
            ms = _time_frame(sc, proxy, tuning)
            table.append({"bvh_width": width, **tuning, "ms": ms})
            if log:
                log(f"autotune width={width} cap={cap} trace={tb} shade={sb}: {ms:.2f} ms")
            if best is None or ms < best["ms"]:
                best = {"bvh_width": width, "tuning": tuning, "ms": ms}
        sc.close()
    best["table"] = table
    return best
