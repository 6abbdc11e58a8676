"""Builds the Lua front-end: the `dort` executable, dort_b200/bin/dort.

The front-end needs the Lua 5.3 interpreter, which this repository does not
contain: it is compiled from a Lua 5.3 source directory given by the caller
(``lua_src``, or the environment variable DORT_LUA_SRC) into
``dort_b200/frontend/_build/liblua.a``.  The executable links that, the
front-end sources in this directory, the embedded Lua modules of
``lua/dort/*.lua`` and the CUDA library ``dort_b200/libdort_gpu.so``
(found next to the package through its run path).

    python -m dort_b200.frontend.build --lua-src <lua 5.3 source dir>
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(HERE, "_build")
EXE = os.path.join(PKG, "bin", "dort")

# the interpreter's sources without its stand-alone programs and the zlib
# binding the reference adds
LUA_SKIP = {"lua.c", "luac.c", "lua_zlib.c"}


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd[:3])}... failed:\n{r.stdout}\n{r.stderr}")


def _newer(out: str, ins) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(i) > t for i in ins)


def _lua_library(lua_src: str) -> str:
    lib = os.path.join(BUILD, "liblua.a")
    srcs = [s for s in sorted(glob.glob(os.path.join(lua_src, "*.c")))
            if os.path.basename(s) not in LUA_SKIP]
    if not srcs:
        raise RuntimeError(f"no Lua sources in {lua_src}")
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, "lua_" + os.path.basename(s) + ".o")
        if _newer(o, [s]):
            _run(["gcc", "-std=gnu99", "-O2", "-fPIC", "-DLUA_USE_POSIX", "-DLUA_COMPAT_5_2",
                  "-c", s, "-o", o])
        objs.append(o)
    if _newer(lib, objs):
        if os.path.exists(lib):
            os.remove(lib)
        _run(["ar", "rcs", lib, *objs])
    return lib


def _embedded_sources() -> str:
    out = os.path.join(BUILD, "lua_sources.cpp")
    files = sorted(glob.glob(os.path.join(HERE, "lua", "dort", "*.lua")))
    lines = ['struct EmbeddedLua { const char* name; const char* source; };',
             'extern const EmbeddedLua kEmbeddedLua[] = {']
    for f in files:
        name = "dort/" + os.path.splitext(os.path.basename(f))[0]
        body = open(f).read()
        assert ")LUA\"" not in body
        lines.append(f'  {{"{name}", R"LUA({body})LUA"}},')
    lines += ['  {nullptr, nullptr},', '};', '']
    text = "\n".join(lines)
    if not os.path.exists(out) or open(out).read() != text:
        with open(out, "w") as fh:
            fh.write(text)
    return out


def build(lua_src: str | None = None, quiet: bool = True) -> str | None:
    """Builds bin/dort; returns its path, or None when no Lua source tree is
    available (the front-end is then skipped)."""
    lua_src = lua_src or os.environ.get("DORT_LUA_SRC")
    if not lua_src or not os.path.exists(os.path.join(lua_src, "lua.h")):
        if not quiet:
            print("Lua 5.3 sources not given (DORT_LUA_SRC): front-end not built")
        return None
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    lib = _lua_library(lua_src)
    srcs = sorted(glob.glob(os.path.join(HERE, "*.cpp"))) + [_embedded_sources()]
    headers = glob.glob(os.path.join(HERE, "*.h")) + [os.path.join(ROOT, "include", "dort_gpu.h")]
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, "fe_" + os.path.basename(s) + ".o")
        if _newer(o, [s, *headers]):
            _run(["g++", "-std=c++17", "-O2", "-Wall", "-I", lua_src, "-I", HERE,
                  "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o])
        objs.append(o)
    gpu_lib = os.path.join(PKG, "libdort_gpu.so")
    if _newer(EXE, [*objs, lib, gpu_lib]):
        _run(["g++", "-o", EXE, *objs, lib, "-L", PKG, "-ldort_gpu",
              "-Wl,-rpath,$ORIGIN/..", "-lm", "-ldl", "-lpthread"])
    if not quiet:
        print(EXE)
    return EXE


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--lua-src", default=None)
    a = ap.parse_args()
    build(a.lua_src, quiet=False)
