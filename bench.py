#!/usr/bin/env python
"""Benchmark of the dort B200 hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dort|reference]
                    [--workload raycast]

Workload "raycast" (the ray-cast kernel configuration): a seeded soup of 1M
random triangles (v0 ~ U[0,1]^3, edges ~ N(0, 0.01)), 16,777,216 rays per
step: 8,388,608 coherent pinhole rays (4096 x 2048 pixel centres) and
8,388,608 diffuse bounce rays (cosine-distributed about the normal at the
first hits of a second pinhole pass), closest hit, fp32.  One step = one ray
cast of all rays.  The rays (512 MB) are larger than L2, so no L2 flush is
needed between steps.

value   rays/s of the device kernel with inputs resident in HBM (CUDA events,
        max over ranks), reported in Mrays/s.
e2e     the same through the C-ABI host entry dort_gpu_raycast with pinned
        host buffers: host->device copy of the rays and device->host copy of
        the hits inside the timed region.
roofline  algorithmic bytes per launch = rays x (32 B ray + 16 B hit +
        N_node x 32 B + N_tri x 36 B), N_node / N_tri = the reference's
        traversal work per ray (its 32-byte binary BVH nodes, 36-byte
        triangles) measured on a sample of the same rays by the CPU leg.
cpu_baseline  the reference's own BVH + triangle code (compiled from its
        sources into oracle/_ref) on all host cores over a bounded sample.

Multi-GPU (torchrun): every rank casts its own 16M rays (weak scaling, no
data exchange); value = all rays / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TRIS = 1_000_000
N_RAYS = 16 * 1024 * 1024
WORKLOAD = "raycast: 1M random tris (SAH BVH), 16M rays (8M coherent pinhole 4096x2048 + 8M diffuse bounce), closest hit"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---- distributed plumbing ------------------------------------------------------

def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ---- clocks ----------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- workload ----------------------------------------------------------------

def raycast_workload(rank: int, caster):
    from dort_b200 import scenes
    verts, tris = scenes.random_triangles(N_TRIS, seed=1)
    coh = scenes.pinhole_rays(4096, 2048)
    dif = scenes.diffuse_rays(verts, tris, N_RAYS - len(coh), caster(verts, tris),
                              seed=2 + 1000 * rank)
    return verts, tris, np.ascontiguousarray(np.concatenate([coh, dif]))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- CPU leg ---------------------------------------------------------------------

def cpu_sample(verts, tris, rays, budget_s: float = 15.0, threads: int | None = None):
    """Reference CPU ray cast (oracle/_ref: the reference's own Bvh + Triangle
    code) on a bounded sample; also the reference's traversal work per ray
    from the oracle restatement on a smaller sample."""
    from oracle import pyoracle as po
    threads = threads or os.cpu_count() or 1
    # interleave coherent and diffuse rays in the sample
    half = len(rays) // 2
    out = {"cores": threads}
    if po.ref_available():
        rb = po.RefBvh(verts, tris, "sah", threads=threads)
        kind = "reference"
        done, t = 0, 0.0
        chunk = 1 << 18
        k = 0
        while t < budget_s and done < len(rays):
            a = (k * chunk // 2) % half
            sample = np.concatenate([rays[a:a + chunk // 2], rays[half + a:half + a + chunk // 2]])
            rb.raycast(sample, threads=threads)
            t += rb.trace_s
            done += len(sample)
            k += 1
        out.update(kind=kind, rays=done, seconds=t)
    else:
        ob = po.OracleBvh(verts, tris, "sah")
        kind = "port"
        t0 = time.perf_counter()
        done = 0
        chunk = 1 << 14
        k = 0
        while time.perf_counter() - t0 < budget_s:
            a = (k * chunk // 2) % half
            sample = np.concatenate([rays[a:a + chunk // 2], rays[half + a:half + a + chunk // 2]])
            ob.raycast(sample)
            done += len(sample)
            k += 1
        out.update(kind=kind, rays=done, seconds=time.perf_counter() - t0, cores=1)
    # traversal work per ray (reference algorithm) on a fixed sample
    ob = po.OracleBvh(verts, tris, "sah")
    idx = np.concatenate([np.arange(0, half, 128), np.arange(half, len(rays), 128)])
    _, _, nodes, tests = ob.raycast(rays[idx], counts=True)
    out["n_node"] = float(nodes.mean())
    out["n_tri"] = float(tests.mean())
    out["work_sample"] = int(len(idx))
    return out


def run_reference(args):
    """--impl reference: the reference's CPU ray cast on this host's cores."""
    from dort_b200 import scenes
    from oracle import pyoracle as po
    threads = os.cpu_count() or 1
    verts, tris = scenes.random_triangles(N_TRIS, seed=1)
    if po.ref_available():
        rb = po.RefBvh(verts, tris, "sah", threads=threads)
        cast = lambda r: rb.raycast(r, threads=threads)
        kind = "reference"
    else:
        ob = po.OracleBvh(verts, tris, "sah")
        cast = lambda r: ob.raycast(r)
        kind = "port"
        threads = 1
    per_step = 1 << 20     # bounded sample of the 16M-ray workload per step
    coh_all = scenes.pinhole_rays(4096, 2048)
    dif = scenes.diffuse_rays(verts, tris, per_step // 2, cast, seed=2)
    stride = len(coh_all) // (per_step // 2)
    sample = np.ascontiguousarray(np.concatenate([coh_all[::stride][:per_step // 2], dif]))
    for _ in range(args.warmup):
        cast(sample)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cast(sample)
    dt = time.perf_counter() - t0
    mrays = len(sample) * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": "Mrays/s", "value": mrays, "unit": "Mrays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "tris": N_TRIS, "rays_per_step": N_RAYS},
        "cpu_baseline": {"value": mrays, "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"{len(sample)} rays per step (1/16 of the workload: "
                                   "every 16th coherent ray + diffuse rays of a smaller "
                                   "second pass), closest hit"},
        "e2e": {"value": mrays, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU leg -----------------------------------------------------------------------

def run_dort(args):
    import torch
    import dort_b200 as db

    rank, world, local, pg = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    def caster(verts, tris):
        sc = db.Scene(verts, tris)
        return lambda r: sc.raycast(r)

    t0 = time.time()
    verts, tris, rays = raycast_workload(rank, caster)
    scene = db.Scene(verts, tris)
    st = scene.stats()
    log(f"[rank {rank}] workload ready in {time.time() - t0:.1f}s; bvh nodes={st['nodes']} "
        f"depth={st['depth']} build={st['build_ms']:.0f}ms")

    n = len(rays)
    d_rays = torch.from_numpy(rays).to(dev)
    d_prim = torch.empty(n, dtype=torch.int32, device=dev)
    d_tb = torch.empty((n, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def step():
        scene.raycast_device(d_rays.data_ptr(), n, d_prim.data_ptr(), d_tb.data_ptr(),
                             stream=sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(pg)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ms_max = max_over_ranks(pg, ms)
    value = world * n * args.steps / (ms_max / 1e3) / 1e6

    # kernel-only duration per launch (events around each launch on its stream)
    per_launch = scene.raycast_timed(d_rays.data_ptr(), n, d_prim.data_ptr(),
                                     d_tb.data_ptr(), stream=sh, repeat=max(3, args.steps))

    # e2e through the host-pointer C-ABI entry with pinned buffers
    h_rays = torch.empty((n, 8), dtype=torch.float32, pin_memory=True)
    h_rays.numpy()[:] = rays
    h_prim = torch.empty(n, dtype=torch.int32, pin_memory=True)
    h_tb = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    import ctypes
    lib = db._abi.lib()

    def e2e_step():
        db._abi.check(lib.dort_gpu_raycast(scene.handle, ctypes.c_void_p(h_rays.data_ptr()),
                                           n, 0, ctypes.c_void_p(h_prim.data_ptr()),
                                           ctypes.c_void_p(h_tb.data_ptr())))
    e2e = None
    if not args.no_e2e:
        e2e_step()
        barrier(pg)
        e2e_steps = min(args.steps, 20)
        te0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        te = time.perf_counter() - te0
        te = max_over_ranks(pg, te)
        e2e = world * n * e2e_steps / te / 1e6

    if rank == 0:
        hbm, peak_kind = peaks()
        cpu = None
        rl = None
        if world == 1 and not args.no_cpu:
            c = cpu_sample(verts, tris, rays)
            cpu = {"value": c["rays"] / c["seconds"] / 1e6, "unit": "Mrays/s",
                   "cores": c["cores"], "kind": c["kind"],
                   "sample": f"{c['rays']} rays interleaved from the coherent and diffuse "
                             f"halves of the workload, {c['seconds']:.1f}s"}
            bytes_per_ray = 32 + 16 + c["n_node"] * 32 + c["n_tri"] * 36
            achieved = n * bytes_per_ray / (per_launch / 1e3) / 1e9
            rl = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                  "frac": achieved / hbm, "traffic": None,
                  "peak_source": peak_kind,
                  "bytes_per_ray": bytes_per_ray, "n_node": c["n_node"], "n_tri": c["n_tri"],
                  "kernel_ms_per_launch": per_launch}
        line = {
            "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tris": N_TRIS, "rays_per_step": n,
                       "l2": "inputs larger than L2 (512 MB of rays per step)",
                       "bvh": f"wide BVH width 8, {st['nodes']} nodes, depth {st['depth']}"},
            "roofline": rl, "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": n * 32,
                    "d2h_bytes_per_step": n * 16},
            "gpu_launches": args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if pg is not None:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dort", choices=["dort", "reference"])
    ap.add_argument("--workload", default="raycast", choices=["raycast"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(args)
        return
    run_dort(args)


if __name__ == "__main__":
    main()
