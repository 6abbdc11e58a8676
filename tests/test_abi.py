"""CPU checks of the C-ABI library: it loads and exports every declared entry
point; argument validation fails cleanly without touching a GPU."""
import ctypes
import os
import re

import numpy as np

import dort_b200 as db
from dort_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(dort_gpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    names = declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_abi_version_and_error_plumbing():
    lib = _abi.lib()
    assert lib.dort_gpu_abi_version() == _abi.ABI_VERSION == 2
    rc = lib.dort_gpu_scene_create(None, None)
    assert rc == -1
    assert b"null" in lib.dort_gpu_last_error()


def test_struct_size_mismatch_rejected():
    h = db.scene_desc(np.zeros((3, 3), np.float32), np.array([[0, 1, 2]], np.uint32))
    h.desc.struct_size = 4
    out = ctypes.c_void_p()
    assert _abi.lib().dort_gpu_scene_create(ctypes.byref(h.desc), ctypes.byref(out)) == -1
    assert b"struct_size" in _abi.lib().dort_gpu_last_error()


def test_bad_vertex_index_rejected_by_host_check():
    v = np.zeros((3, 3), np.float32)
    t = np.array([[0, 1, 7]], np.uint32)
    try:
        db.host_check_raycast(v, t, np.zeros((1, 8), np.float32))
    except db.DortError as e:
        assert e.status == -1 and "vertex" in str(e)
    else:
        raise AssertionError("expected DortError")


def test_non_finite_vertex_rejected():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, np.nan, 0]], np.float32)
    t = np.array([[0, 1, 2]], np.uint32)
    try:
        db.host_check_raycast(v, t, np.zeros((1, 8), np.float32))
    except db.DortError as e:
        assert "finite" in str(e)
    else:
        raise AssertionError("expected DortError")


def test_ctypes_layouts_match_the_header(tmp_path):
    """The ctypes mirror has the C compiler's size and field offsets for every
    structure of include/dort_gpu.h."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        import pytest
        pytest.skip("gcc not available")
    structs = {"dort_material": _abi.Material, "dort_shape": _abi.Shape,
               "dort_light": _abi.Light, "dort_scene_desc": _abi.SceneDesc,
               "dort_camera": _abi.Camera, "dort_render_params": _abi.RenderParams,
               "dort_wavefront_tuning": _abi.WavefrontTuning, "dort_batch_job": _abi.BatchJob}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dort_gpu.h"',
             'int main(void) {']
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([gcc, "-I", inc, str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run(
        [str(exe)], check=True, capture_output=True, text=True).stdout.split("\n") if l)
    for cname, cls in structs.items():
        assert int(out[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)
