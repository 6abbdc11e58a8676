"""PLY ingest (CPU): dort_b200.ply / builder and the Lua front-end's reader
against the reference's reader (read_ply_to_mesh over rply,
src/dort/ply_mesh.cpp), pinned by tests/golden/ply_golden.npz (files of
tests/golden/ply_cases.py and the reference's points and triangles for each,
written by tests/golden/gen_ply_golden.py)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ply_cases  # noqa: E402
import pyoracle  # noqa: E402
from dort_b200 import builder as b  # noqa: E402
from dort_b200 import ply  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "ply_golden.npz"))
NAMES = sorted({k.split("/")[0] for k in GOLDEN.files})
DORT = os.path.join(ROOT, "dort_b200", "bin", "dort")
needs_frontend = pytest.mark.skipif(not os.path.exists(DORT), reason="front-end not built")


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("ply")
    out = {}
    for name in NAMES:
        path = str(d / (name + ".ply"))
        with open(path, "wb") as f:
            f.write(GOLDEN[name + "/file"].tobytes())
        out[name] = path
    return out


def test_fixture_files_are_the_generated_cases():
    cases = ply_cases.cases()
    assert sorted(cases) == NAMES
    for name, data in cases.items():
        assert GOLDEN[name + "/file"].tobytes() == data, name


@pytest.mark.parametrize("name", NAMES)
def test_reader_matches_the_reference(files, name):
    pts, verts = ply.read_ply(files[name])
    assert pts.dtype == np.float32
    assert np.array_equal(pts.view(np.uint32), GOLDEN[name + "/points"].view(np.uint32)), name
    assert np.array_equal(verts, GOLDEN[name + "/vertices"].astype(np.int64)), name


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference harness not built")
def test_reference_reader_still_gives_the_fixture(files):
    for name in NAMES:
        pts, verts = pyoracle.ref_read_ply(files[name])
        assert np.array_equal(pts.view(np.uint32), GOLDEN[name + "/points"].view(np.uint32))
        assert np.array_equal(verts, GOLDEN[name + "/vertices"])


def test_reader_errors(tmp_path, files):
    with pytest.raises(OSError, match="Could not open ply mesh file for reading"):
        ply.read_ply(str(tmp_path / "missing.ply"))
    data = open(files["ble_large_triangles"], "rb").read()
    cut = tmp_path / "cut.ply"
    cut.write_bytes(data[:len(data) // 2])
    with pytest.raises(ply.PlyError, match="Could not read ply file"):
        ply.read_ply(str(cut))
    if pyoracle.ref_available():
        with pytest.raises(ValueError):
            pyoracle.ref_read_ply(str(cut))
    # an index past the points: the reference reads it without complaint and
    # would index out of bounds later; refused here
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\n"
                    b"property float y\nproperty float z\nelement face 1\n"
                    b"property list uchar int vertex_indices\nend_header\n"
                    b"0 0 0\n1 0 0\n0 1 0\n3 0 1 7\n")
    with pytest.raises(ply.PlyError, match="out of range"):
        ply.read_ply(str(bad))


def _builder_scene(path, transform):
    B = b.Builder()
    B.set_material(b.lambert_material(b.rgb(0.6)))
    B.set_transform(transform)
    B.add_read_ply_mesh(path)
    B.set_transform(b.translate(0, 0, 1))
    B.add_ply_mesh(b.read_ply_mesh(path))
    return B.build_scene()


def test_builder_adds_ply_triangles_under_its_transform(files):
    t = b.translate(1, 2, 3) * b.rotate_y(0.3) * b.scale(2, 1, 0.5)
    for name in NAMES:
        d = _builder_scene(files[name], t)
        pts = GOLDEN[name + "/points"].astype(np.float64)
        idx = GOLDEN[name + "/vertices"].astype(np.int64)
        first = t.apply_points(pts)[idx]
        second = (t * b.translate(0, 0, 1)).apply_points(pts)[idx]
        want = np.concatenate([first, second]).astype(np.float32)
        assert d["verts"].shape == want.shape, name
        np.testing.assert_allclose(d["verts"], want, rtol=1e-6, atol=1e-5, err_msg=name)
        assert np.array_equal(d["tris"].reshape(-1), np.arange(len(want))), name
        assert len(d["tri_material"]) == len(want) // 3


@needs_frontend
def test_frontend_reads_like_the_builder(tmp_path, files):
    script = tmp_path / "ply_scene.lua"
    lines = ["local b, g = dort.builder, dort.geometry",
             "local B = b.make()",
             "b.set_material(B, dort.material.make_lambert { albedo = dort.spectrum.rgb(0.6) })",
             "b.set_transform(B, g.translate(1, 2, 3) * g.rotate_y(0.3) * g.scale(2, 1, 0.5))",
             "local path = dort.env.get_argv()[1]",
             "b.add_read_ply_mesh(B, path)",
             "b.set_transform(B, g.translate(0, 0, 1))",
             "b.add_ply_mesh(B, dort.shape.read_ply_mesh(path))",
             "b.build_scene(B)"]
    script.write_text("\n".join(lines) + "\n")
    t = b.translate(1, 2, 3) * b.rotate_y(0.3) * b.scale(2, 1, 0.5)
    for name in NAMES:
        rec = tmp_path / (name + ".json")
        out = subprocess.run([DORT, str(script), files[name]], capture_output=True, text=True,
                             env=dict(os.environ, DORT_LUA_RECORD=str(rec)), timeout=120)
        assert out.returncode == 0, out.stderr
        lua = json.load(open(rec))
        py = _builder_scene(files[name], t)
        lv = np.asarray(lua["verts"], np.float32).reshape(-1, 3)
        assert lv.shape == py["verts"].shape, name
        # the two transform the float points in double and round once; the
        # bound is a few float ulps of the largest coordinate
        scale = float(np.abs(py["verts"]).max()) if py["verts"].size else 1.0
        np.testing.assert_allclose(lv, py["verts"], rtol=0, atol=4e-7 * scale + 1e-7,
                                   err_msg=name)
        assert np.array_equal(np.asarray(lua["tris"]).reshape(-1, 3), py["tris"]), name


@needs_frontend
def test_frontend_ply_errors(tmp_path, files):
    data = open(files["ble_large_triangles"], "rb").read()
    cut = tmp_path / "cut.ply"
    cut.write_bytes(data[:len(data) // 2])
    for path, msg in ((str(tmp_path / "missing.ply"), "Could not open ply mesh file for reading"),
                      (str(cut), "Could not read ply file")):
        script = tmp_path / "read.lua"
        script.write_text(f'dort.shape.read_ply_mesh("{path}")\n')
        out = subprocess.run([DORT, str(script)], capture_output=True, text=True, timeout=60)
        assert out.returncode == 1 and msg in out.stderr, out.stderr
