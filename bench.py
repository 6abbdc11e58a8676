#!/usr/bin/env python
"""Benchmark of the dort B200 hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dort|reference]
                    [--workload pt1080p|raycast|batch|adjoint|cornell] [--spp S]
                    [--converged-spp C] [--no-sub] [--no-cpu] [--no-e2e]
                    [--renderer pt|lt|bdpt] [--engine megakernel|wavefront]

Workload "pt1080p" (default; the wavefront configuration): 1920x1080, 256
samples per pixel, max depth 16, a 1,997,122-triangle scene (geodesic
icosphere of frequency 316 displaced by fBm of amplitude 0.1, plus a
2-triangle ground plane; seeded mix of Lambert / GGX conductor / dielectric
materials) lit by a procedural 1024x512 HDR sky.  One step = one frame.
value   samples/s of the wavefront renderer (one CUDA graph per frame),
        CUDA events on the launch stream, max over ranks.
config.megakernel_samples_per_s  the plain per-pixel megakernel on the same
        frame; both draw the same random numbers per pixel and sample.
config.equal_rmse  the error of both 256-spp frames against a converged
        frame of the same scene: C samples per pixel (default 20,480), half
        rendered by each renderer as 256-spp frames with independent seeds,
        every frame accumulated in float64 on the host (FP64 CPU
        accumulation).  Relative RMSE = sqrt(mean((x - r)^2)) / mean(r) over
        all pixels and channels, with the converged frame's own variance (from
        the spread of its frames) subtracted; the spp each renderer needs for
        1 %.  at_1pct: each renderer's own half (C/2 spp, below 1 % error),
        the device seconds it took and the ratio of those times: the samples/s
        ratio at equal RMSE below 1 %, measured.
e2e     the wavefront frame through the C-ABI host entry
        dort_gpu_render_wavefront, image copied back to host memory; the
        scene's creation through dort_gpu_scene_create (what a script pays
        once before its first frame) is reported beside it.
roofline  the extend (closest-hit) stage: algorithmic bytes = rays x (32 B
        ray + 16 B hit + the reference traversal's N_node x 32 B + N_tri x
        36 B measured on a sample of this workload's rays).
sub     the other workloads of the metric, measured in the same run at N=1:
        the ray cast (Mrays/s), the batch (samples/s) and the adjoint (ms),
        each the line its own --workload prints (fewer steps).

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

Workloads "batch" (64 seeded scenes of 10k-500k random triangles in one
wavefront launch, samples/s), "adjoint" (512x512, 64 spp, depth 6, 500k
triangles: forward + backward ms) and "cornell" (the Cornell box at 256x256,
64 spp, depth 8, with --renderer pt / lt / bdpt and, for pt, --engine
megakernel / wavefront; samples/s) print their own lines; the first two are
also the pt1080p line's sub-records.

Multi-GPU (torchrun): every rank renders its own frame or casts its own 16M
rays (weak scaling, no data exchange); value = all units / max-over-ranks
time.  The converged frame, the CPU baseline and the sub-records run at N=1
only.
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
# DRAM bytes (read + write) of one raycast_kernel launch over the 16M-ray
# workload, from the ncu capture summarised in
# profiles/raycast_kernel_1Mtri_16Mrays.md (dram__bytes_read.sum +
# dram__bytes_write.sum); reported as the roofline's traffic.
RAYCAST_TRAFFIC_BYTES = 800.7e6
# The bound that applies to the ray cast beside the HBM roofline (whose
# algorithmic bytes count the reference's binary-tree work, more than the
# wide tree does, so its frac exceeds 1): issue slots.  Figures of one
# launch under ncu --set full (profiles/raycast_kernel_1Mtri_16Mrays.md).
RAYCAST_LIMITER = {
    "bound": "issue slots (divergent traversal)",
    "source": "ncu --set full of one raycast_kernel launch, "
              "profiles/raycast_kernel_1Mtri_16Mrays.md",
    "issue_slots_busy": 0.739, "simt_efficiency": 11.6 / 32, "achieved_occupancy": 0.496,
    "dram_throughput": 0.013,
    "top_stall": "long_scoreboard, 3.85 cycles per issue",
}
WORKLOAD = "raycast: 1M random tris (SAH BVH), 16M rays (8M coherent pinhole 4096x2048 + 8M diffuse bounce), closest hit"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---- distributed plumbing ------------------------------------------------------

def dist_setup(n_gpus: int):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE).  The
    process group runs over NCCL; DORT_DIST_BACKEND=gloo runs the same
    plumbing on CPU processes (the multi-rank tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = os.environ.get("DORT_DIST_BACKEND", "nccl")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's shard: every rank renders or casts its own
    independent work (weak scaling, no data-path exchange)."""
    return base + 1000 * rank


def job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return world * units_per_rank / seconds_max


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
                              seed=rank_seed(2, rank))
    return verts, tris, np.ascontiguousarray(np.concatenate([coh, dif]))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def classify_watertight(prim_mt, tb_mt, prim_wt, tb_wt, eps: float = 1e-4) -> dict:
    """The rays on which the watertight test and the reference's
    Moller-Trumbore disagree, by kind: a ray that slips through an edge under
    one test, a tie in t between two triangles (a shared edge), or nearer
    hits at an edge; 'unexplained' counts the rest (none expected)."""
    miss = 0xFFFFFFFF
    near = lambda tb: np.minimum(np.minimum(tb[:, 1], tb[:, 2]), 1 - tb[:, 1] - tb[:, 2]) < eps
    d = prim_mt != prim_wt
    mt_miss, wt_miss = d & (prim_mt == miss), d & (prim_wt == miss)
    both = d & ~mt_miss & ~wt_miss
    tie = both & (np.abs(tb_mt[:, 0] - tb_wt[:, 0]) <= 1e-5 * np.abs(tb_wt[:, 0]))
    out = {"rays": int(len(prim_mt)), "ids_differ": int(d.sum()),
           "mt_slips_at_edge": int((mt_miss & near(tb_wt)).sum()),
           "watertight_misses_mt_edge_hit": int((wt_miss & near(tb_mt)).sum()),
           "same_t_other_triangle": int(tie.sum()),
           "nearer_hit_at_edge": int((both & ~tie & (near(tb_mt) | near(tb_wt))).sum())}
    out["unexplained"] = out["ids_differ"] - sum(
        out[k] for k in ("mt_slips_at_edge", "watertight_misses_mt_edge_hit",
                         "same_t_other_triangle", "nearer_hit_at_edge"))
    return out


def host_info() -> dict:
    """The host's logical core count and CPU model (the CPU baseline's box)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"host_cores": os.cpu_count(), "cpu_model": model}


def ref_procs(per_proc_gb: float = 0.6) -> int:
    """Single-threaded reference processes for the CPU baseline: one per
    logical core, fewer if half the available memory cannot hold them (each
    holds the 2M-triangle scene and its reference BVH, about 0.4 GB)."""
    n = os.cpu_count() or 1
    try:
        import psutil
        avail_gb = psutil.virtual_memory().available / 2**30
        n = max(1, min(n, int(avail_gb * 0.5 / per_proc_gb)))
    except Exception:  # noqa: BLE001 -- psutil missing: all cores
        pass
    return n


class Ctx:
    """Rank, world size, local device and process group of this process."""

    def __init__(self, rank, world, local, pg):
        self.rank, self.world, self.local, self.pg = rank, world, local, pg


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
                         **host_info(),
                         "sample": f"{len(sample)} rays per step (1/16 of the workload: "
                                   "every 16th coherent ray + diffuse rays of a smaller "
                                   "second pass), closest hit"},
        "e2e": {"value": mrays, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU leg -----------------------------------------------------------------------

def measure_raycast(args, ctx, steps, warmup, cpu_budget=15.0, e2e_steps=20):
    """The ray-cast workload; returns its JSON line on rank 0 (else None)."""
    import torch
    import dort_b200 as db

    rank, world, local, pg = ctx.rank, ctx.world, ctx.local, ctx.pg
    dev = torch.device("cuda", local)

    def caster(verts, tris):
        sc = db.Scene(verts, tris)
        return lambda r: sc.raycast(r)

    t0 = time.time()
    verts, tris, rays = raycast_workload(rank, caster)
    scene = db.Scene(verts, tris, bvh_build=args.bvh_build)
    st = scene.stats()
    log(f"[rank {rank}] workload ready in {time.time() - t0:.1f}s; bvh nodes={st['nodes']} "
        f"depth={st['depth']} build={st['build_ms']:.0f}ms ({st['bvh_build']} BVH "
        f"{st['bvh_ms']:.0f}ms)")

    n = len(rays)
    d_rays = torch.from_numpy(rays).to(dev)
    d_prim = torch.empty(n, dtype=torch.int32, device=dev)
    d_tb = torch.empty((n, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def step():
        scene.raycast_device(d_rays.data_ptr(), n, d_prim.data_ptr(), d_tb.data_ptr(),
                             stream=sh)

    for _ in range(warmup):
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
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ms_max = max_over_ranks(pg, ms)
    value = job_rate(n * steps, world, ms_max / 1e3) / 1e6

    # kernel-only duration per launch (events around each launch on its stream)
    per_launch = scene.raycast_timed(d_rays.data_ptr(), n, d_prim.data_ptr(),
                                     d_tb.data_ptr(), stream=sh, repeat=max(3, steps))

    # the watertight test (DORT_SCENE_WATERTIGHT) on the same rays: its rate
    # and every ray on which it disagrees with the reference's test, by kind
    wt = None
    if world == 1 and not args.no_cpu:
        wsc = db.Scene(verts, tris, bvh_build=args.bvh_build, watertight=True)
        w_prim = torch.empty_like(d_prim)
        w_tb = torch.empty_like(d_tb)
        w_ms = wsc.raycast_timed(d_rays.data_ptr(), n, w_prim.data_ptr(), w_tb.data_ptr(),
                                 stream=sh, repeat=max(3, steps))
        torch.cuda.synchronize()
        wt = classify_watertight(d_prim.cpu().numpy().view(np.uint32), d_tb.cpu().numpy(),
                                 w_prim.cpu().numpy().view(np.uint32), w_tb.cpu().numpy())
        wt["mrays_per_s"] = n / (w_ms / 1e3) / 1e6
        wsc.close()

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
        e2e_steps = max(1, min(steps, e2e_steps))
        te0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        te = time.perf_counter() - te0
        te = max_over_ranks(pg, te)
        e2e = world * n * e2e_steps / te / 1e6

    line = None
    if rank == 0:
        hbm, peak_kind = peaks()
        cpu = None
        rl = None
        if world == 1 and not args.no_cpu:
            c = cpu_sample(verts, tris, rays, budget_s=cpu_budget)
            cpu = {"value": c["rays"] / c["seconds"] / 1e6, "unit": "Mrays/s",
                   "cores": c["cores"], "kind": c["kind"], **host_info(),
                   "sample": f"{c['rays']} rays interleaved from the coherent and diffuse "
                             f"halves of the workload, {c['seconds']:.1f}s"}
            bytes_per_ray = 32 + 16 + c["n_node"] * 32 + c["n_tri"] * 36
            achieved = n * bytes_per_ray / (per_launch / 1e3) / 1e9
            rl = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                  "frac": achieved / hbm, "traffic": RAYCAST_TRAFFIC_BYTES,
                  "traffic_source": "ncu capture of one launch "
                                    "(profiles/raycast_kernel_1Mtri_16Mrays.md)",
                  "peak_source": peak_kind,
                  "bytes_per_ray": bytes_per_ray, "n_node": c["n_node"], "n_tri": c["n_tri"],
                  "kernel_ms_per_launch": per_launch,
                  "frac_note": "algorithmic bytes are the reference's binary-BVH work per "
                               "ray; the 8-wide tree visits fewer nodes, so frac can exceed "
                               "1; the applicable bound is in limiter",
                  "measured_dram_gbs": RAYCAST_TRAFFIC_BYTES / (per_launch / 1e3) / 1e9,
                  "limiter": RAYCAST_LIMITER}
        line = {
            "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": ms_max / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tris": N_TRIS, "rays_per_step": n,
                       "l2": "inputs larger than L2 (512 MB of rays per step)",
                       "bvh": f"wide BVH width 8, {st['nodes']} nodes, depth {st['depth']}",
                       "bvh_build": st["bvh_build"], "bvh_build_ms": round(st["bvh_ms"], 2),
                       "watertight": wt},
            "roofline": rl, "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": n * 32,
                    "d2h_bytes_per_step": n * 16},
            "gpu_launches": steps,
            "clocks": clk,
        }
    scene.close()
    return line if rank == 0 else None


# ---- pt1080p workload ------------------------------------------------------------

PT_W, PT_H, PT_SPP, PT_DEPTH = 1920, 1080, 256, 16
PT_WORKLOAD = ("pt1080p: wavefront path tracing 1920x1080, 256 spp, max depth 16, "
               "1,997,122-tri fBm-displaced icosphere + ground plane, Lambert / GGX conductor / "
               "dielectric mix, procedural 1024x512 HDR sky")
REF_SAMPLE_W, REF_SAMPLE_H = 480, 270
# DRAM bytes (read + write) of one wf_extend launch over a full queue
# (4,194,304 rays, waves 6-8 of the 16-spp frame), mean of three launches of
# the ncu capture summarised in profiles/wf_extend_pt1080p.md: 777 MB, 185 B
# per ray; reported as the roofline's traffic.
EXTEND_TRAFFIC_BYTES = 730.4e6
EXTEND_TRAFFIC_RAYS = 4194304
# The bound that applies to the extension stage beside the HBM roofline:
# issue slots and latency.  Figures of one wf_extend launch under
# ncu --set full (profiles/wf_extend_pt1080p.md): smsp__issue_active,
# smsp__thread_inst_executed_per_inst_executed / 32, sm__warps_active,
# lts__throughput and gpu__dram_throughput as fractions of their peaks.
EXTEND_LIMITER = {
    "bound": "issue slots and node-fetch latency (divergent traversal)",
    "source": "ncu --set full of one full-queue wf_extend launch, "
              "profiles/wf_extend_pt1080p.md",
    "issue_slots_busy": 0.668, "simt_efficiency": 11.92 / 32, "achieved_occupancy": 0.534,
    "occupancy_limit": 0.5625, "l2_throughput": 0.178, "dram_throughput": 0.072,
    "top_stall": "long_scoreboard (L1/L2 node and stack loads), 6.02 cycles per issue",
}

_ref_worker_scene = None


def _ref_worker_init():
    global _ref_worker_scene
    from dort_b200 import scenes
    from oracle import pyoracle as po
    _ref_worker_scene = po.RefPtScene(scenes.wavefront_scene(), threads=1)


def _ref_worker_render(seed):
    img, secs = _ref_worker_scene.render(REF_SAMPLE_W, REF_SAMPLE_H, 1, max_depth=PT_DEPTH,
                                         seed=seed, threads=1)
    return secs


def ref_pt_pool(procs):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    return ctx.Pool(procs, initializer=_ref_worker_init)


def ref_pt_step(pool, procs, step):
    t0 = time.perf_counter()
    pool.map(_ref_worker_render, [1000 * step + k for k in range(procs)])
    return time.perf_counter() - t0


def pt_reference_work(sd, n=1 << 15):
    """The reference traversal's work per ray (binary middle-split BVH over the
    frame's triangles, its dort default) on primary + one-bounce diffuse rays
    of the frame, from the oracle's restatement of that traversal."""
    from dort_b200 import scenes
    from oracle import pyoracle as po
    ob = po.OracleBvh(sd["verts"], sd["tris"], "middle")
    side = int(np.sqrt(n))
    cam = scenes.camera_rays(sd["camera"], side * 16 // 9, side * 9 // 16)
    prim, tb = ob.raycast(cam)
    hit, pos, nrm, t = scenes.hit_frames(sd["verts"], sd["tris"], cam, prim, tb)
    rng = np.random.default_rng(7)
    d = scenes.cosine_dirs(nrm, rng)
    sec = np.zeros((len(pos), 8), np.float32)
    sec[:, 0:3] = pos
    sec[:, 3] = np.abs(np.float32(1e-3) * t)
    sec[:, 4:7] = d
    sec[:, 7] = np.inf
    rays = np.concatenate([cam, sec])
    _, _, nodes, tests = ob.raycast(rays, counts=True)
    return float(nodes.mean()), float(tests.mean()), len(rays)


def converged_halves(sc, sd, W, H, frames_each, frame_spp, d_out, sh, stream, tuning):
    """The converged frame of the scene, rendered half by each renderer: each
    renders `frames_each` frames of `frame_spp` samples per pixel with
    independent seeds (CUDA events around every frame), each frame is copied
    to the host and accumulated in float64.  Returns per renderer its mean
    image, the variance of that mean per pixel (from the spread of its
    frames), its spp and device seconds; and the mean and variance of all
    frames together (the reference)."""
    import torch
    import dort_b200 as db
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    halves = {}
    tot = np.zeros((H, W, 3), np.float64)
    tot2 = np.zeros((H, W, 3), np.float64)
    for name, seed0 in (("wavefront", 2_000_000), ("megakernel", 1_000_000)):
        acc = np.zeros((H, W, 3), np.float64)
        acc2 = np.zeros((H, W, 3), np.float64)
        ms = 0.0
        for k in range(frames_each):
            p = db.render_params(sd["camera"], W, H, frame_spp, max_depth=PT_DEPTH,
                                 seed=seed0 + k)
            ev0.record(stream)
            if name == "wavefront":
                sc.render_wavefront_device(p, d_out.data_ptr(), stream=sh, tuning=tuning)
            else:
                sc.render_device(p, d_out.data_ptr(), stream=sh)
            ev1.record(stream)
            ev1.synchronize()
            ms += ev0.elapsed_time(ev1)
            img = d_out.view(H, W, 3).cpu().numpy().astype(np.float64)
            acc += img
            acc2 += img * img
        mean = acc / frames_each
        var_frame = np.maximum(acc2 / frames_each - mean * mean, 0.0) * frames_each / (
            frames_each - 1)
        halves[name] = {"mean": mean, "var_mean": var_frame / frames_each,
                        "spp": frames_each * frame_spp, "seconds": ms / 1e3}
        tot += acc
        tot2 += acc2
    n = 2 * frames_each
    ref = tot / n
    var_ref = np.maximum(tot2 / n - ref * ref, 0.0) * n / (n - 1) / n
    return halves, ref, var_ref


def equal_rmse(frames: dict, ref, var_ref, ref_spp: int, spp: int, rates: dict,
               halves: dict | None = None, pixels: int = 0) -> dict:
    """Relative RMSE of each frame against the converged one (its own
    variance subtracted), the spp each renderer needs for 1 %, and the
    samples/s ratio at equal RMSE; with `halves` (each renderer's own
    converged half), the error each half reaches and the time it took."""
    mref = float(ref.mean())
    vref = float(var_ref.mean())
    out = {"reference": f"{ref_spp} spp, half rendered by each renderer as independent "
                        f"{spp}-spp frames, float64 accumulation on the host",
           "reference_spp": ref_spp,
           "reference_rel_rmse": float(np.sqrt(vref) / mref),
           "target_rel_rmse": 0.01}
    need = {}
    for name, x in frames.items():
        raw = float(((x.astype(np.float64) - ref) ** 2).mean())
        rel = float(np.sqrt(max(raw - vref, 0.0)) / mref)
        out[f"rel_rmse_{name}"] = rel
        out[f"rel_rmse_{name}_uncorrected"] = float(np.sqrt(raw) / mref)
        # Monte Carlo error falls as 1/sqrt(spp)
        need[name] = int(np.ceil(spp * (rel / 0.01) ** 2))
        out[f"spp_for_1pct_{name}"] = need[name]
    # the expected error of one frame from the reference's own spread
    out["rel_rmse_expected_from_spread"] = float(np.sqrt(vref * ref_spp / spp) / mref)
    # both renderers trace the same paths (same random numbers), so equal spp
    # is equal RMSE
    out["equal_rmse_spp"] = max(spp, max(need.values()))
    out["wavefront_over_megakernel_at_equal_rmse"] = rates["wavefront"] / rates["megakernel"]
    if halves:
        at = {}
        for name, h in halves.items():
            at[name] = {"spp": h["spp"], "seconds": round(h["seconds"], 3),
                        "samples_per_s": pixels * h["spp"] / h["seconds"] if pixels else None,
                        "rel_rmse": float(np.sqrt(h["var_mean"].mean()) / mref)}
        a, b = halves["wavefront"], halves["megakernel"]
        at["rel_rmse_between"] = float(np.sqrt(((a["mean"] - b["mean"]) ** 2).mean()) / mref)
        at["rel_rmse_between_expected"] = float(
            np.sqrt((a["var_mean"] + b["var_mean"]).mean()) / mref)
        at["wavefront_over_megakernel"] = b["seconds"] / a["seconds"]
        out["at_1pct"] = at
    return out


def measure_pt(args, ctx):
    """The 1080p wavefront frame; returns its JSON line on rank 0."""
    import torch
    import dort_b200 as db
    from dort_b200 import scenes

    rank, world, local, pg = ctx.rank, ctx.world, ctx.local, ctx.pg
    dev = torch.device("cuda", local)
    t0 = time.time()
    sd = scenes.wavefront_scene()
    sd["bvh_build"] = args.bvh_build
    tc0 = time.perf_counter()
    sc = db.scene_from_dict(sd)
    scene_create_ms = (time.perf_counter() - tc0) * 1e3
    st = sc.stats()
    log(f"[rank {rank}] scene ready in {time.time() - t0:.1f}s; nodes={st['nodes']} "
        f"depth={st['depth']} create={scene_create_ms:.0f}ms ({st['bvh_build']} BVH "
        f"{st['bvh_ms']:.0f}ms)")
    spp = args.spp or PT_SPP
    p = db.render_params(sd["camera"], PT_W, PT_H, spp, max_depth=PT_DEPTH,
                         seed=rank_seed(42, rank))
    # the fixed tuning: 2^25 path slots (about 11 GB of path state), fewer,
    # fuller waves (at 256 spp 2^22 / 2^23 / 2^24 / 2^25 slots measured
    # 567 / 592 / 606 / 616 M samples/s), blocks of 128; by default the
    # autotuner times its candidates (this one among them) on this frame first
    tuning = {"queue_capacity": 1 << 25, "trace_block": 128, "shade_block": 128,
              "sort_rays": args.sort_rays == "on", "stage_queues": args.stage_queues == "on"}
    if args.queue_capacity:
        tuning["queue_capacity"] = args.queue_capacity
    tuned = None
    if args.tuning == "auto" and not args.queue_capacity:
        from dort_b200 import autotune as at
        tuned = at.tune_scene(sc, p, budget_s=30.0)
        tuning.update(tuned["tuning"])
        log(f"[rank {rank}] autotune: {tuned['tuning']} ({tuned['candidates']} candidates, "
            f"{tuned['seconds']:.1f}s)")
    d_out = torch.empty(PT_H * PT_W * 3, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    samples = PT_W * PT_H * spp

    def frame():
        sc.render_wavefront_device(p, d_out.data_ptr(), stream=sh, tuning=tuning)

    for _ in range(args.warmup):
        frame()
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
        frame()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ms_max = max_over_ranks(pg, ms)
    value = job_rate(samples * args.steps, world, ms_max / 1e3)
    wf_img = d_out.view(PT_H, PT_W, 3).cpu().numpy()

    # the plain per-pixel megakernel on the same frame
    mega_steps = max(1, min(args.steps, 3))
    sc.render_device(p, d_out.data_ptr(), stream=sh)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(mega_steps):
        sc.render_device(p, d_out.data_ptr(), stream=sh)
    ev1.record(stream)
    torch.cuda.synchronize()
    mega_ms = max_over_ranks(pg, ev0.elapsed_time(ev1) / mega_steps)
    mega_img = d_out.view(PT_H, PT_W, 3).cpu().numpy()
    mega_value = world * samples / (mega_ms / 1e3)

    # per-stage times of one frame (events around each stage, no graph)
    stages = sc.wavefront_stage_times(p, tuning)

    e2e = None
    if not args.no_e2e:
        img, _ = sc.render_wavefront(p, tuning)      # warm the host path
        barrier(pg)
        e2e_steps = max(1, min(args.steps, 3))
        te0 = time.perf_counter()
        for _ in range(e2e_steps):
            img, _ = sc.render_wavefront(p, tuning)
        te = max_over_ranks(pg, time.perf_counter() - te0)
        e2e = world * samples * e2e_steps / te

    # equal RMSE: both 256-spp frames against a converged frame, and each
    # renderer timed to its own converged half (N=1 only)
    eq = None
    if world == 1 and args.converged_spp > 0:
        frames_each = max(2, args.converged_spp // (2 * PT_SPP))
        halves, ref, var_ref = converged_halves(sc, sd, PT_W, PT_H, frames_each, PT_SPP, d_out,
                                                sh, stream, tuning)
        eq = equal_rmse({"wavefront": wf_img, "megakernel": mega_img}, ref, var_ref,
                        2 * frames_each * PT_SPP, spp,
                        {"wavefront": value, "megakernel": mega_value}, halves, PT_W * PT_H)
        at = eq["at_1pct"]
        log(f"[rank {rank}] converged frame {2 * frames_each * PT_SPP} spp: 256-spp rel RMSE "
            f"{eq['rel_rmse_wavefront']:.4f}; {at['wavefront']['spp']} spp: wavefront "
            f"{at['wavefront']['seconds']:.1f}s rel RMSE {at['wavefront']['rel_rmse']:.4f}, "
            f"megakernel {at['megakernel']['seconds']:.1f}s rel RMSE "
            f"{at['megakernel']['rel_rmse']:.4f}")

    line = None
    if rank == 0:
        rr_between = float(np.sqrt(((wf_img.astype(np.float64) - mega_img) ** 2).mean())
                           / max(float(mega_img.mean()), 1e-30))
        hbm, peak_kind = peaks()
        rl = None
        cpu = None
        rays_per_frame = stages["rays"]
        if world == 1 and not args.no_cpu:
            n_node, n_tri, nwork = pt_reference_work(sd)
            procs = ref_procs()
            pool = ref_pt_pool(procs)
            ref_pt_step(pool, procs, 0)                  # builds + warms the workers
            secs = ref_pt_step(pool, procs, 1)
            pool.close()
            cpu_value = procs * REF_SAMPLE_W * REF_SAMPLE_H / secs
            cpu = {"value": cpu_value, "unit": "samples/s", "cores": procs, "kind": "reference",
                   **host_info(),
                   "sample": f"{procs} single-threaded reference PathRenderer processes (one "
                             f"per logical core), each one {REF_SAMPLE_W}x{REF_SAMPLE_H} frame "
                             f"at 1 spp of the same scene and camera ({secs:.1f}s); GGX "
                             "conductor timed as Phong"}
            # dominant stage: the extend (closest-hit) stage, over the frame's
            # extension rays (counted by the staged run)
            ext_rays = stages["extend_rays"]
            bytes_per_ray = 32 + 16 + n_node * 32 + n_tri * 36
            achieved = ext_rays * bytes_per_ray / (stages["extend"] / 1e3) / 1e9
            cap = tuning["queue_capacity"]
            rl = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                  "frac": achieved / hbm,
                  # per full-queue launch of this run's capacity: the captured
                  # bytes per ray times the rays of such a launch (the
                  # traffic grows with the rays a launch traces)
                  "traffic": EXTEND_TRAFFIC_BYTES / EXTEND_TRAFFIC_RAYS * cap,
                  "traffic_source": f"ncu capture of full-queue launches of "
                                    f"{EXTEND_TRAFFIC_RAYS} rays "
                                    f"(profiles/wf_extend_pt1080p.md), scaled to "
                                    f"{cap} rays",
                  "traffic_bytes_per_ray": EXTEND_TRAFFIC_BYTES / EXTEND_TRAFFIC_RAYS,
                  "algorithmic_bytes_per_full_launch": cap * bytes_per_ray,
                  "peak_source": peak_kind,
                  "kernel": "wf_extend (closest hit)", "bytes_per_ray": bytes_per_ray,
                  "frac_note": "algorithmic bytes are the reference's binary-BVH work per "
                               "ray (its 32-byte nodes and 36-byte triangles); the 8-wide "
                               "tree visits fewer nodes and stays L2-resident, so frac can "
                               "reach 1 without DRAM doing so: measured_dram_gbs is the "
                               "stage's real DRAM rate, limiter the bound that applies",
                  "n_node": n_node, "n_tri": n_tri, "work_sample_rays": nwork,
                  "extend_rays_per_frame": ext_rays,
                  # the same stage against the DRAM traffic it really moves
                  # (the tree is L2-resident): measured bytes per ray over the
                  # stage time
                  "measured_dram_gbs": ext_rays * EXTEND_TRAFFIC_BYTES / EXTEND_TRAFFIC_RAYS
                                       / (stages["extend"] / 1e3) / 1e9,
                  "stage_ms_per_frame": {k: stages[k] for k in
                                         ("regen", "extend", "shade", "shadow", "neeb")},
                  "limiter": EXTEND_LIMITER}
        line = {
            "metric": "samples/s at 1080p equal-RMSE, wavefront vs plain GPU",
            "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": PT_WORKLOAD, "width": PT_W, "height": PT_H, "spp": spp,
                       "max_depth": PT_DEPTH, "tris": int(st["tris"]),
                       "megakernel_samples_per_s": mega_value,
                       "wavefront_over_megakernel": value / mega_value,
                       "rel_rmse_wavefront_vs_megakernel": rr_between,
                       "equal_rmse": eq,
                       "rays_per_frame": rays_per_frame,
                       "mrays_per_s": rays_per_frame * args.steps * world / (ms_max / 1e3) / 1e6,
                       "queue_capacity": tuning["queue_capacity"],
                       "trace_block": tuning["trace_block"],
                       "shade_block": tuning["shade_block"],
                       "tuning": "fixed" if args.queue_capacity else args.tuning,
                       "autotune": tuned,
                       "sort_rays": tuning["sort_rays"],
                       "stage_queues": tuning["stage_queues"],
                       "extend_rays_per_frame": stages["extend_rays"],
                       "stage_ms_per_frame": {k: round(stages[k], 3) for k in
                                              ("regen", "extend", "shade", "shadow", "neeb")},
                       "bvh_build": st["bvh_build"], "bvh_build_ms": round(st["bvh_ms"], 2),
                       # about 330 bytes of path state and queues per slot
                       "l2": "frame state (path queues ~%.0f GB, image 25 MB) larger than L2"
                             % (tuning["queue_capacity"] * 330 / 1e9)},
            "roofline": rl, "cpu_baseline": cpu,
            # per frame the caller passes its render parameters and reads the
            # image back; the scene (vertices, indices, materials, sky) goes to
            # the device once, at dort_gpu_scene_create
            "e2e": {"value": e2e, "unit": "samples/s",
                    "h2d_bytes_per_step": ctypes_sizeof_params(),
                    "d2h_bytes_per_step": PT_W * PT_H * 12,
                    "scene_create_ms": round(scene_create_ms, 1),
                    "scene_h2d_bytes": scene_input_bytes(sd),
                    "scene_device_bytes": int(st["device_bytes"])},
            "gpu_launches": args.steps * int(stages["waves"] * 6 + 2),
            "clocks": clk,
        }
    sc.close()
    return line


def ctypes_sizeof_params() -> int:
    import ctypes
    from dort_b200 import _abi
    return ctypes.sizeof(_abi.RenderParams)


def scene_input_bytes(sd: dict) -> int:
    """Bytes of the host arrays a scene description hands to
    dort_gpu_scene_create."""
    n = 0
    for k in ("verts", "tris", "tri_material", "tri_emission", "sky_rgb"):
        v = sd.get(k)
        if v is not None:
            n += int(np.asarray(v).nbytes)
    return n


def run_reference_pt(args):
    procs = ref_procs()
    pool = ref_pt_pool(procs)
    for w in range(args.warmup):
        ref_pt_step(pool, procs, w)
    secs = 0.0
    for k in range(args.steps):
        secs += ref_pt_step(pool, procs, 100 + k)
    pool.close()
    value = procs * REF_SAMPLE_W * REF_SAMPLE_H * args.steps / secs
    line = {
        "impl": "reference", "metric": "samples/s at 1080p equal-RMSE, wavefront vs plain GPU",
        "value": value, "unit": "samples/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": PT_WORKLOAD, "width": PT_W, "height": PT_H, "spp": PT_SPP,
                   "max_depth": PT_DEPTH},
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": procs,
                         "kind": "reference", **host_info(),
                         "sample": f"per step {procs} single-threaded reference PathRenderer "
                                   f"processes each render one {REF_SAMPLE_W}x{REF_SAMPLE_H} "
                                   "1-spp frame of the same scene and camera (the reference's "
                                   "thread pool crashes intermittently above 1 thread); GGX "
                                   "conductor timed as Phong"},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- batch workload -----------------------------------------------------------------

BATCH_WORKLOAD = ("batch: 64 seeded jobs, random-triangle soups of 10k-500k tris (log-uniform) "
                  "with one quad light, resolution 64-1024 per axis (log-uniform), spp 16-512, "
                  "depth 8-16, one wavefront launch (one CUDA graph) for all jobs")


def measure_batch(args, ctx, steps, warmup, mega_warmup=True):
    """The batch workload; returns its JSON line on rank 0."""
    import torch
    import dort_b200 as db
    from dort_b200 import scenes

    rank, world, local, pg = ctx.rank, ctx.world, ctx.local, ctx.pg
    t0 = time.time()
    specs = scenes.batch_jobs(count=64, seed=rank_seed(4, rank))
    jobs = []
    t_create = time.time()
    for k, (sd, w, h, spp, depth) in enumerate(specs):
        sd["bvh_build"] = args.bvh_build
        sc = db.scene_from_dict(sd)
        jobs.append((sc, db.render_params(sd["camera"], w, h, spp, max_depth=depth, seed=k)))
    create_s = time.time() - t_create
    bvh_ms = sum(sc.stats()["bvh_ms"] for sc, _ in jobs)
    built = jobs[0][0].stats()["bvh_build"]
    samples = sum(w * h * spp for (_, w, h, spp, _) in specs)
    log(f"[rank {rank}] 64 scenes ready in {time.time() - t0:.1f}s ({create_s:.2f}s to create, "
        f"{built} BVH builds {bvh_ms:.0f} ms), {samples / 1e9:.2f}G samples")
    # the batch tuning: 2^22 slots, or the autotuner's choice on a proxy
    # batch (every job at an eighth of its samples) with --tuning auto in a
    # batch run of its own
    tuning = {"queue_capacity": args.queue_capacity or 1 << 22,
              "sort_rays": args.sort_rays == "on"}
    tuned = None
    if args.tuning == "auto" and args.workload == "batch":
        from dort_b200 import autotune as at
        tuned = at.tune_batch(jobs, budget_s=60.0)
        tuning.update(tuned["tuning"])
        log(f"[rank {rank}] batch autotune: {tuned['tuning']} ({tuned['seconds']:.1f}s)")
    b = db.Batch(jobs, tuning)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        b.render(stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        b.render(stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(pg)
    ms = max_over_ranks(pg, ev0.elapsed_time(ev1))
    clk = clocks.stop()
    st = b.stats()
    value = world * samples * steps / (ms / 1e3)
    # the plain per-pixel megakernel, one launch per job
    outs = [torch.empty(p.width * p.height * 3, dtype=torch.float32, device="cuda")
            for _, p in jobs]
    if mega_warmup:
        for (sc, p), o in zip(jobs, outs):
            sc.render_device(p, o.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
    ev0.record(stream)
    for (sc, p), o in zip(jobs, outs):
        sc.render_device(p, o.data_ptr(), stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    mega_ms = max_over_ranks(pg, ev0.elapsed_time(ev1))
    line = None
    if rank == 0:
        line = {
            "metric": "batched samples/s, wavefront batch vs per-job megakernel", "value": value,
            "unit": "samples/s", "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "jobs": len(jobs), "samples": samples,
                       "megakernel_samples_per_s": world * samples / (mega_ms / 1e3),
                       "batch_over_megakernel": (mega_ms / (ms / steps)),
                       "rays_per_batch": st["rays"], "waves": st["waves"],
                       "queue_capacity": tuning["queue_capacity"], "autotune": tuned,
                       "bvh_build": built, "bvh_build_ms_total": round(bvh_ms, 1),
                       "scene_create_s_total": round(create_s, 3)},
            "roofline": None, "cpu_baseline": None,
            "e2e": None, "gpu_launches": steps * int(st["waves"] * 6 + 2), "clocks": clk,
        }
    b.close()
    for sc, _ in jobs:
        sc.close()
    return line


# ---- adjoint workload ---------------------------------------------------------------

ADJ_WORKLOAD = ("adjoint: 512x512, 64 spp, depth 6, 500k random tris with per-triangle RGB "
                "albedo U(0.1,0.9) and 8 emissive tris; L2 loss vs a seeded target; forward "
                "render + path-replay backward for albedo and emission gradients")


def measure_adjoint(args, ctx, steps, warmup):
    """The adjoint workload; returns its JSON line on rank 0."""
    import torch
    import dort_b200 as db
    from dort_b200 import scenes

    rank, world, local, pg = ctx.rank, ctx.world, ctx.local, ctx.pg
    sd = scenes.adjoint_scene()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 512, 512, 64, max_depth=6, seed=rank_seed(1, rank))
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(9)
    target = sc.adjoint_forward(p, np.clip(alb * rng.uniform(0.8, 1.2, alb.shape), 0, 1)
                                .astype(np.float32), em)

    def step():
        img = sc.adjoint_forward(p, alb, em)
        loss, g = db.loss_l2(img, target)
        return sc.adjoint_backward(p, g, alb, em)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    dt = max_over_ranks(pg, time.perf_counter() - t0)
    clk = clocks.stop()
    # the step's parts, timed apart after the timed steps (host clock, each
    # call returns host arrays): forward render, loss, backward
    img = sc.adjoint_forward(p, alb, em)
    loss, g = db.loss_l2(img, target)
    parts = {}
    for name, fn in (("forward", lambda: sc.adjoint_forward(p, alb, em)),
                     ("loss", lambda: db.loss_l2(img, target)),
                     ("backward", lambda: sc.adjoint_backward(p, g, alb, em))):
        torch.cuda.synchronize()
        tp = time.perf_counter()
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        parts[name] = round((time.perf_counter() - tp) / 2 * 1e3, 2)
    line = None
    if rank == 0:
        ms = dt / steps * 1e3
        line = {
            "metric": "adjoint ms (forward + backward, host arrays)", "value": ms, "unit": "ms",
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": ADJ_WORKLOAD, "tris": int(len(sd["tris"])),
                       "parts_ms": parts},
            "roofline": None, "cpu_baseline": None,
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": int(2 * alb.nbytes * 2 +
                                                                          512 * 512 * 12 * 2),
                    "d2h_bytes_per_step": int(alb.nbytes * 2 + 512 * 512 * 12)},
            "gpu_launches": steps * 4, "clocks": clk,
        }
    sc.close()
    return line


C1_W, C1_H, C1_SPP, C1_DEPTH = 256, 256, 64, 8
C1_WORKLOAD = ("cornell: Cornell box (10 wall tris, two 12-tri boxes, 0.5 x 0.5 quad light), "
               "256x256, 64 spp, max depth 8")


def measure_cornell(args, ctx, steps, warmup):
    """The Cornell-box configuration (256 x 256, 64 spp, depth 8) with the
    renderer --renderer names: pt (the megakernel, or --engine wavefront),
    lt or bdpt; device output, CUDA events; returns its JSON line on rank 0."""
    import torch
    import dort_b200 as db
    from dort_b200 import scenes

    rank, world, local, pg = ctx.rank, ctx.world, ctx.local, ctx.pg
    dev = torch.device("cuda", local)
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], C1_W, C1_H, C1_SPP, max_depth=C1_DEPTH,
                         seed=rank_seed(42, rank), renderer=args.renderer)
    d_out = torch.empty(C1_W * C1_H * 3, dtype=torch.float32, device=dev)
    sh = torch.cuda.current_stream(dev).cuda_stream
    wavefront = args.renderer == "pt" and args.engine == "wavefront"

    def frame():
        if wavefront:
            sc.render_wavefront_device(p, d_out.data_ptr(), sh)
        else:
            sc.render_device(p, d_out.data_ptr(), sh)

    for _ in range(warmup):
        frame()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        frame()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(pg, e0.elapsed_time(e1) / 1e3) * 1e3
    clk = clocks.stop()
    img = d_out.view(C1_H, C1_W, 3).cpu().numpy()
    line = None
    if rank == 0:
        samples = C1_W * C1_H * C1_SPP * steps * world
        line = {
            "metric": "samples/s", "value": samples / (ms / 1e3), "unit": "samples/s",
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": C1_WORKLOAD, "renderer": args.renderer,
                       "engine": "wavefront" if wavefront else "megakernel",
                       "image_mean": float(img.mean()),
                       "l2": "inputs are a few KB (L2-resident by design of the workload)"},
            "roofline": None, "cpu_baseline": None, "e2e": None,
            # kernels per frame: kernel + resolve (pt megakernel, lt); bdpt: per
            # chunk of 2^20 samples the light and camera walks, four connection
            # cases and the gather, then the resolve; the wavefront's graph is
            # not counted
            "gpu_launches": (None if wavefront else steps * (
                2 if args.renderer != "bdpt" else
                7 * -(-(C1_W * C1_H * C1_SPP) // (1 << 20)) + 1)),
            "clocks": clk,
        }
    sc.close()
    return line


def run_dort(args):
    """The GPU arm: one process per GPU; rank 0 prints one JSON line."""
    import torch
    rank, world, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    ctx = Ctx(rank, world, local, pg)
    if args.workload == "pt1080p":
        line = measure_pt(args, ctx)
        if world == 1 and not args.no_sub:
            # the metric's other parts, fewer steps each, after the frame
            sub = {}
            for name, fn in (("raycast", lambda: measure_raycast(args, ctx, 20, 3, cpu_budget=8.0,
                                                                 e2e_steps=5)),
                             ("adjoint", lambda: measure_adjoint(args, ctx, 3, 3)),
                             ("batch", lambda: measure_batch(args, ctx, 1, 1,
                                                             mega_warmup=False))):
                t0 = time.time()
                sub[name] = fn()
                log(f"[rank {rank}] sub-record {name} in {time.time() - t0:.0f}s")
                torch.cuda.empty_cache()
            if line is not None:
                line["sub"] = sub
    elif args.workload == "batch":
        line = measure_batch(args, ctx, args.steps, args.warmup)
    elif args.workload == "adjoint":
        line = measure_adjoint(args, ctx, args.steps, args.warmup)
    elif args.workload == "cornell":
        line = measure_cornell(args, ctx, args.steps, args.warmup)
    else:
        line = measure_raycast(args, ctx, args.steps, args.warmup)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0,
                    help="timed steps (default: 5 for pt1080p, 100 for raycast)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dort", choices=["dort", "reference"])
    ap.add_argument("--workload", default="pt1080p",
                    choices=["pt1080p", "raycast", "batch", "adjoint", "cornell"])
    ap.add_argument("--renderer", default="pt", choices=["pt", "lt", "bdpt"],
                    help="cornell workload: the renderer")
    ap.add_argument("--engine", default="megakernel", choices=["megakernel", "wavefront"],
                    help="cornell workload with the pt renderer: megakernel or wavefront")
    ap.add_argument("--spp", type=int, default=0, help="pt1080p samples per pixel (default 256)")
    ap.add_argument("--converged-spp", type=int, default=20480,
                    help="pt1080p: samples per pixel of the converged frame, half rendered "
                         "by each renderer (0: skip)")
    ap.add_argument("--no-sub", action="store_true",
                    help="pt1080p: skip the ray-cast, adjoint and batch sub-records")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--tuning", default="auto", choices=["auto", "fixed"],
                    help="wavefront tuning: the autotuner's choice on the frame, or the "
                         "fixed 2^25 slots / 128-thread blocks")
    ap.add_argument("--queue-capacity", type=int, default=0,
                    help="pt1080p, batch: path slots of the wavefront (implies a fixed tuning; "
                         "small values keep a profiled run's device memory small)")
    ap.add_argument("--stage-queues", default="off", choices=["on", "off"],
                    help="stage the shadow queue through bulk copies (TMA) into shared memory")
    ap.add_argument("--sort-rays", default="off", choices=["on", "off"],
                    help="sort each wave's extension rays (wavefront)")
    ap.add_argument("--bvh-build", default=None, choices=["host", "device", "ploc"],
                    help="where scenes build their BVH (default: the library's, the device)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps <= 0:
        args.steps = {"pt1080p": 5, "raycast": 100, "batch": 2, "adjoint": 5,
                      "cornell": 20}[args.workload]
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        if args.workload in ("raycast",):
            run_reference(args)
        elif args.workload == "pt1080p":
            run_reference_pt(args)
        else:
            why = ("the reference has no batched or adjoint renderer"
                   if args.workload in ("batch", "adjoint") else
                   "the reference arm times the pt1080p and raycast workloads only")
            print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    run_dort(args)


if __name__ == "__main__":
    main()
