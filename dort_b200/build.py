"""Builds the in-tree CUDA library ``dort_b200/libdort_gpu.so`` for sm_100a.

Every ``csrc/*.cu`` / ``csrc/*.cpp`` is compiled by nvcc into ``_build/`` and
linked into one shared library that exports the C ABI of
``include/dort_gpu.h``.  Objects are rebuilt when a source or header is newer.

    python -m dort_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libdort_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max([os.path.getmtime(h) for h in hs] + [0.0])


def _compile(src: str, ptxas_verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    hm = _headers_mtime()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hm):
        return obj, ""
    cmd = [nvcc(), *ARCH, *COMMON, "-c", src, "-o", obj]
    if ptxas_verbose and src.endswith(".cu"):
        cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(ptxas_verbose: bool = False, quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_verbose), srcs))
    objs = [o for o, _ in results]
    if ptxas_verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static",
               "-Xcompiler", "-fPIC", "-Xlinker", "--no-undefined", "-lpthread",
               "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    build(ptxas_verbose=a.verbose_ptxas, quiet=False)
