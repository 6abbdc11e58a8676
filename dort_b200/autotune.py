"""Autotuner for the wavefront renderer.

The search itself is native (dort_gpu_autotune_wavefront /
dort_gpu_autotune_batch, csrc/autotune.cu): block sizes of the trace and
shade stages ranked on a proxy frame of the caller's scene and camera, path
slot capacities 2^22 .. 2^28 on the frame itself, each candidate timed with
CUDA events.  This module adds the one choice that needs the scene rebuilt,
the BVH node width, by tuning each width's scene and keeping the fastest.

    best = autotune(scene_dict, params)   # {"bvh_width": 8, "tuning": {...}, "ms": ...}
    sc = scene_from_dict(scene_dict, bvh_width=best["bvh_width"])
    sc.render_wavefront(params, best["tuning"])
"""
from __future__ import annotations

import ctypes
import time

from . import _abi, scene_from_dict

DEFAULT_WIDTHS = (8,)


def _as_dict(t: _abi.WavefrontTuning) -> dict:
    return {"queue_capacity": int(t.queue_capacity), "trace_block": int(t.trace_block),
            "shade_block": int(t.shade_block)}


def tune_scene(scene, params: _abi.RenderParams, budget_s: float = 30.0) -> dict:
    """Native search on one scene handle: {"tuning", "ms", "candidates",
    "seconds", "cut"}."""
    t = _abi.WavefrontTuning()
    st = (ctypes.c_double * 4)()
    _abi.check(_abi.lib().dort_gpu_autotune_wavefront(scene.handle, ctypes.byref(params),
                                                       budget_s * 1e3, ctypes.byref(t), st))
    return {"tuning": _as_dict(t), "ms": st[1], "candidates": int(st[0]),
            "seconds": st[2] / 1e3, "cut": bool(st[3])}


def tune_batch(jobs, budget_s: float = 60.0) -> dict:
    """Native search for a batch (a list of (Scene, RenderParams))."""
    arr = (_abi.BatchJob * len(jobs))()
    for i, (sc, p) in enumerate(jobs):
        arr[i].scene = sc.handle
        arr[i].params = p
    t = _abi.WavefrontTuning()
    st = (ctypes.c_double * 4)()
    _abi.check(_abi.lib().dort_gpu_autotune_batch(arr, len(jobs), budget_s * 1e3,
                                                   ctypes.byref(t), st))
    return {"tuning": _as_dict(t), "ms": st[1], "candidates": int(st[0]),
            "seconds": st[2] / 1e3, "cut": bool(st[3])}


def autotune(scene: dict, params: _abi.RenderParams, widths=DEFAULT_WIDTHS,
             budget_s: float = 60.0, log=None) -> dict:
    """Returns {"bvh_width", "tuning", "ms", "table"}: the fastest BVH width
    with its native tuning (each width gets an equal share of the budget)."""
    table = []
    best = None
    t0 = time.perf_counter()
    for width in widths:
        left = budget_s - (time.perf_counter() - t0)
        if best is not None and left <= 0:
            break
        sc = scene_from_dict(scene, bvh_width=width)
        try:
            r = tune_scene(sc, params, max(left / max(1, len(widths)), 1.0))
        finally:
            sc.close()
        table.append({"bvh_width": width, **r})
        if log:
            log(f"autotune width={width}: {r['tuning']} {r['ms']:.2f} ms")
        if best is None or r["ms"] < best["ms"]:
            best = {"bvh_width": width, "tuning": r["tuning"], "ms": r["ms"]}
    best["table"] = table
    return best
