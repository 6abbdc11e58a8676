"""The Lua front-end (dort_b200/bin/dort, dort_b200/frontend/).

CPU: scene scripts written for the reference renderer run through the
front-end in record mode (the flattened scene is written as JSON instead of
being sent to the GPU), and every scene must equal what dort_b200.builder
makes of the same scene, as restated in tests/golden/ref_scenes.py.  Run on
the reference's own test scripts when its test directory is available.

GPU: a scene script renders through the front-end and the image equals the
Python API's render of the same scene with the same seed.
"""
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
sys.path.insert(0, HERE)

import ref_scenes  # noqa: E402

DORT = os.path.join(ROOT, "dort_b200", "bin", "dort")
# the reference's test scripts: DORT_REFERENCE_TESTS, else the test/ folder of
# DORT_REFERENCE_TREE or of a "reference" checkout beside this repository
REFERENCE_TESTS = os.environ.get("DORT_REFERENCE_TESTS") or os.path.join(
    os.environ.get("DORT_REFERENCE_TREE") or os.path.join(os.path.dirname(ROOT), "reference"),
    "test")

needs_frontend = pytest.mark.skipif(not os.path.exists(DORT),
                                    reason="front-end not built (needs Lua 5.3 sources)")


def _mat_key(m):
    param = (list(m["param"]) + [0.0] * 4)[:4]
    return (int(m["kind"]), tuple(np.round(np.float32(m["color"]), 6)),
            tuple(np.round(np.float32(m["color2"]), 6)), tuple(np.round(np.float32(param), 6)))


def _compare(lua: dict, py: dict, name: str):
    """Flat scenes equal up to float rounding; materials compared by value."""
    close = dict(rtol=1e-5, atol=1e-5)
    lv = np.asarray(lua["verts"], np.float32).reshape(-1, 3)
    pv = np.asarray(py["verts"], np.float32).reshape(-1, 3)
    assert lv.shape == pv.shape, name
    np.testing.assert_allclose(lv, pv, err_msg=name, **close)
    assert np.array_equal(np.asarray(lua["tris"]).reshape(-1, 3), py["tris"]), name
    lm = [_mat_key(lua["materials"][i]) for i in lua["tri_material"]]
    pm = [_mat_key(py["materials"][i]) for i in py["tri_material"]]
    assert lm == pm, name
    np.testing.assert_allclose(np.asarray(lua["tri_emission"], np.float32).reshape(-1, 3),
                               py["tri_emission"], err_msg=name, **close)
    assert ("tri_light_verts" in lua) == ("tri_light_verts" in py), name
    if "tri_light_verts" in py:
        np.testing.assert_allclose(np.asarray(lua["tri_light_verts"], np.float32).reshape(-1, 9),
                                   py["tri_light_verts"], err_msg=name, **close)
    assert len(lua["shapes"]) == len(py["shapes"]), name
    for a, b in zip(lua["shapes"], py["shapes"]):
        assert a["kind"] == b["kind"], name
        assert _mat_key(lua["materials"][a["material"]]) == _mat_key(py["materials"][b["material"]])
        np.testing.assert_allclose(a["param"], (list(b["param"]) + [0] * 4)[:4], err_msg=name, **close)
        np.testing.assert_allclose(a["to_world"], b["to_world"], err_msg=name, **close)
        np.testing.assert_allclose(a["emission"], b["emission"], err_msg=name, **close)
        assert ("light_to_world" in a) == (b.get("light_to_world") is not None), name
        if "light_to_world" in a:
            np.testing.assert_allclose(a["light_to_world"], b["light_to_world"], err_msg=name, **close)
    assert len(lua["delta_lights"]) == len(py["delta_lights"]), name
    for a, b in zip(lua["delta_lights"], py["delta_lights"]):
        assert a["kind"] == b["kind"], name
        np.testing.assert_allclose(a["rgb"], b["rgb"], err_msg=name, **close)
        np.testing.assert_allclose(a["vec"], b["vec"], err_msg=name, **close)
    np.testing.assert_allclose(lua["sky_const"], py.get("sky_const", (0, 0, 0)), err_msg=name, **close)
    lc, pc = lua["camera"], py["camera"]
    assert lc["kind"] == pc.get("kind", 0), name
    for k in ("origin", "right", "up", "forward"):
        np.testing.assert_allclose(lc[k], pc[k], err_msg=name, **close)
    for k in ("fov", "lens_radius", "focal_distance", "dimension"):
        assert abs(lc[k] - pc.get(k, 0.0)) <= 1e-5 * max(1.0, abs(pc.get(k, 0.0))), (name, k)


@needs_frontend
@pytest.mark.skipif(not os.path.isdir(REFERENCE_TESTS), reason="reference test scripts absent")
def test_reference_test_scripts_record_like_the_python_builder(tmp_path):
    env = dict(os.environ, DORT_LUA_RECORD=str(tmp_path / "s%d.json"))
    out = subprocess.run(
        [DORT, os.path.join(HERE, "lua", "record_reference_tests.lua"), "test",
         "test_box", "test_simple", "test_bsdf"],
        cwd=os.path.dirname(REFERENCE_TESTS), env=env, capture_output=True, text=True,
        timeout=300)
    assert out.returncode == 0, out.stderr
    scene_of = {}
    for line in out.stdout.splitlines():
        sid, name = line.split(None, 1)
        scene_of[name.strip()] = int(sid)
    checked = 0
    for case in ref_scenes.CASES:
        if case["name"] not in scene_of:
            continue
        lua = json.load(open(tmp_path / f"s{scene_of[case['name']]}.json"))
        _compare(lua, ref_scenes.build(case), case["name"])
        checked += 1
    assert checked >= 80


SCENE_LUA = r'''
local _ENV = require "dort/dsl"
local scene = define_scene(function()
  local white = lambert_material { albedo = rgb(0.7) }
  material(white)
  local m = mesh {
    points = { point(-4, 0, -4), point(4, 0, -4), point(4, 0, 4), point(-4, 0, 4) },
    vertices = { 0, 1, 2,  0, 2, 3 },
  }
  add_triangle(m, 0)
  add_triangle(m, 3)
  block(function()
    material(phong_material { albedo = rgb(0.4, 0.3, 0.2), exponent = 30 })
    transform(translate(-1, 1, 0) * rotate_y(0.5))
    add_shape(cube())
  end)
  block(function()
    material(dielectric_material { ior_inside = 1.5 })
    transform(translate(1.5, 1, 0.5))
    add_shape(sphere { radius = 1 })
  end)
  block(function()
    transform(look_at(point(0, 5, -2), point(0, 0, 0), vector(0, 1, 0)))
    add_diffuse_light { shape = disk { radius = 1 }, radiance = rgb(8) }
  end)
  add_light(point_light { point = point(3, 4, -3), intensity = rgb(20) })
  add_light(infinite_light { radiance = rgb(0.2) })
  camera(pinhole_camera {
    transform = look_at(point(0, 3, -8), point(0, 1, 0), vector(0, 1, 0)) * scale(1, -1, 1),
    fov = 0.8,
  })
end)
local image = render(scene, { hdr = true, x_res = 96, y_res = 64, iterations = 16,
  max_depth = 4, sampler = random_sampler { seed = 7 } })
write_rgbe_image(dort.env.get_argv()[1], image)
'''


def _python_scene():
    from dort_b200 import builder as b
    B = b.Builder()
    B.set_material(b.lambert_material(b.rgb(0.7)))
    m = B.mesh([b.point(-4, 0, -4), b.point(4, 0, -4), b.point(4, 0, 4), b.point(-4, 0, 4)],
               [0, 1, 2, 0, 2, 3])
    B.add_triangle(m, 0)
    B.add_triangle(m, 3)

    def cube_block():
        B.set_material(b.phong_material(b.rgb(0.4, 0.3, 0.2), exponent=30))
        B.set_transform(b.translate(-1, 1, 0) * b.rotate_y(0.5))
        B.add_shape(b.cube())
    B.block(cube_block)

    def ball():
        B.set_material(b.dielectric_material(ior_inside=1.5))
        B.set_transform(b.translate(1.5, 1, 0.5))
        B.add_shape(b.sphere(1))
    B.block(ball)

    def lamp():
        B.set_transform(b.look_at(b.point(0, 5, -2), b.point(0, 0, 0), b.vector(0, 1, 0)))
        B.add_diffuse_light(b.disk(1), b.rgb(8))
    B.block(lamp)
    B.add_light(B.point_light(b.point(3, 4, -3), b.rgb(20)))
    B.add_light(b.infinite_light(b.rgb(0.2)))
    B.set_camera(b.pinhole_camera(
        b.look_at(b.point(0, 3, -8), b.point(0, 1, 0), b.vector(0, 1, 0)) * b.scale(1, -1, 1),
        fov=0.8))
    return B.build_scene()


@needs_frontend
def test_own_script_records_like_the_python_builder(tmp_path):
    script = tmp_path / "scene.lua"
    script.write_text(SCENE_LUA)
    env = dict(os.environ, DORT_LUA_RECORD=str(tmp_path / "rec.json"))
    out = subprocess.run([DORT, str(script), str(tmp_path / "img.hdr")], env=env,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    _compare(json.load(open(tmp_path / "rec.json")), _python_scene(), "own scene")


@needs_frontend
def test_frontend_reports_unknown_parameters(tmp_path):
    script = tmp_path / "bad.lua"
    script.write_text('local m = dort.material.make_lambert { albedo = dort.spectrum.rgb(1), '
                      'albdo = 2 }\n')
    out = subprocess.run([DORT, str(script)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 1
    assert "Unused parameter 'albdo'" in out.stderr


@needs_frontend
@pytest.mark.gpu
def test_script_renders_like_the_python_api(tmp_path, cuda):
    import dort_b200 as db
    from dort_b200.image import read_rgbe, rgbe_quantize
    script = tmp_path / "scene.lua"
    script.write_text(SCENE_LUA)
    out = subprocess.run([DORT, str(script), str(tmp_path / "img.hdr")], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lua_img = read_rgbe(str(tmp_path / "img.hdr"))
    d = _python_scene()
    sc = db.scene_from_dict(d)
    p = db.render_params(d["camera"], 96, 64, 16, max_depth=4, seed=7)
    py_img = rgbe_quantize(sc.render_wavefront(p)[0])
    sc.close()
    # same scene, same seed, same renderer: the same image up to the float
    # rounding of the two flattenings' vertex transforms
    diff = np.abs(lua_img.astype(np.float64) - py_img)
    assert float(diff.mean()) < 1e-3 * max(float(py_img.mean()), 1e-6), float(diff.mean())


@needs_frontend
@pytest.mark.gpu
@pytest.mark.parametrize("renderer", ["lt", "bdpt"])
def test_script_renders_other_renderers_like_the_python_api(tmp_path, cuda, renderer):
    import dort_b200 as db
    from dort_b200.image import read_rgbe, rgbe_quantize
    script = tmp_path / "scene.lua"
    script.write_text(SCENE_LUA.replace("max_depth = 4,", f'max_depth = 4, renderer = "{renderer}",'))
    out = subprocess.run([DORT, str(script), str(tmp_path / "img.hdr")], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lua_img = read_rgbe(str(tmp_path / "img.hdr"))
    d = _python_scene()
    sc = db.scene_from_dict(d)
    p = db.render_params(d["camera"], 96, 64, 16, max_depth=4, seed=7, renderer=renderer)
    py_img = rgbe_quantize(sc.render(p)[0])
    sc.close()
    # same sample streams; splats are summed by float atomics in any order
    diff = np.abs(lua_img.astype(np.float64) - py_img)
    assert float(diff.mean()) < 1e-3 * max(float(py_img.mean()), 1e-6), float(diff.mean())


@needs_frontend
def test_frontend_bdpt_debug_images_are_refused(tmp_path):
    script = tmp_path / "scene.lua"
    script.write_text(SCENE_LUA.replace(
        "max_depth = 4,", 'max_depth = 4, renderer = "bdpt", debug_image_dir = "x",'))
    env = dict(os.environ, DORT_LUA_RECORD=str(tmp_path / "rec.json"))
    out = subprocess.run([DORT, str(script), str(tmp_path / "img.hdr")], env=env,
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    assert "debug_image_dir" in out.stderr


ADJOINT_LUA = r'''
local _ENV = require "dort/dsl"
local scene = define_scene(function()
  material(lambert_material { albedo = rgb(0.7, 0.6, 0.5) })
  local floor = mesh {
    points = { point(-4, 0, -4), point(4, 0, -4), point(4, 0, 4), point(-4, 0, 4) },
    vertices = { 0, 1, 2,  0, 2, 3 },
  }
  add_triangle(floor, 0)
  add_triangle(floor, 3)
  block(function()
    material(lambert_material { albedo = rgb(0.3, 0.5, 0.7) })
    local wall = mesh {
      points = { point(-3, 0, 2), point(3, 0, 2), point(3, 4, 3), point(-3, 4, 3) },
      vertices = { 0, 1, 2,  0, 2, 3 },
    }
    add_triangle(wall, 0)
    add_triangle(wall, 3)
  end)
  block(function()
    material(lambert_material { albedo = rgb(0) })
    local lamp = mesh {
      points = { point(1, 4, -1), point(1, 4, 1), point(-1, 4, 1), point(-1, 4, -1) },
      vertices = { 2, 1, 0,  3, 2, 0 },
    }
    for _, index in ipairs({0, 3}) do
      local shape = triangle(lamp, index)
      local light = diffuse_light { radiance = rgb(10, 9, 8), shape = shape }
      add_light(light)
      add_shape(shape, light)
    end
  end)
  camera(pinhole_camera {
    transform = look_at(point(0, 3, -8), point(0, 1, 0), vector(0, 1, 0)) * scale(1, -1, 1),
    fov = 0.8,
  })
end)
local job = dort.render.make(scene, { x_res = 48, y_res = 32, iterations = 8, max_depth = 4,
  sampler = random_sampler { seed = 7 } })
local albedo, emission = dort.render.triangle_params(scene)
local target = dort.render.adjoint_forward(job, { albedo = dort.image.axpy(-0.2, albedo, albedo) })
local image = dort.render.adjoint_forward(job, { albedo = albedo })
local loss, dl_dimage = dort.render.loss_l2(image, target)
local d_albedo, d_emission = dort.render.adjoint_backward(job,
  { dl_dimage = dl_dimage, albedo = albedo })
local out = dort.env.get_argv()[1]
dort.image.write_pfm(out .. "/image.pfm", image)
dort.image.write_pfm(out .. "/d_albedo.pfm", d_albedo)
dort.image.write_pfm(out .. "/d_emission.pfm", d_emission)
dort.image.write_pfm(out .. "/albedo.pfm", albedo)
print(string.format("loss %.9g", loss))
'''


def _scene_from_record(rec: dict) -> dict:
    """The Python scene dict of a recorded flat scene (triangles only)."""
    cam = rec["camera"]
    return {"verts": np.asarray(rec["verts"], np.float32).reshape(-1, 3),
            "tris": np.asarray(rec["tris"], np.uint32).reshape(-1, 3),
            "tri_material": np.asarray(rec["tri_material"], np.uint32),
            "materials": [{"kind": m["kind"], "color": tuple(m["color"]),
                           "color2": tuple(m["color2"]), "param": tuple(m["param"])}
                          for m in rec["materials"]],
            "tri_emission": np.asarray(rec["tri_emission"], np.float32).reshape(-1, 3),
            "camera": {"origin": cam["origin"], "right": cam["right"], "up": cam["up"],
                       "forward": cam["forward"], "fov": cam["fov"], "kind": cam["kind"]}}


@needs_frontend
def test_adjoint_script_records_and_refuses_without_a_gpu(tmp_path):
    """In record mode (no GPU) the script's scene records, its per-triangle
    parameters come out, and the adjoint itself stops with a clear error."""
    script = tmp_path / "adjoint.lua"
    script.write_text(ADJOINT_LUA)
    env = dict(os.environ, DORT_LUA_RECORD=str(tmp_path / "rec.json"))
    out = subprocess.run([DORT, str(script), str(tmp_path)], env=env, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 1
    assert "the adjoint needs a GPU" in out.stderr
    sd = _scene_from_record(json.load(open(tmp_path / "rec.json")))
    assert len(sd["tris"]) == 6 and sd["tri_emission"][4:].min() > 0


@needs_frontend
@pytest.mark.gpu
def test_script_adjoint_matches_the_python_api(tmp_path, cuda):
    import dort_b200 as db
    from dort_b200.image import read_pfm
    script = tmp_path / "adjoint.lua"
    script.write_text(ADJOINT_LUA)
    # the flat scene, recorded without GPU work (the adjoint calls then stop
    # the script, after define_scene, which is all the record needs)
    env = dict(os.environ, DORT_LUA_RECORD=str(tmp_path / "rec.json"))
    subprocess.run([DORT, str(script), str(tmp_path)], env=env, capture_output=True, text=True,
                   timeout=120)
    rec = json.load(open(tmp_path / "rec.json"))
    out = subprocess.run([DORT, str(script), str(tmp_path)], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    lua_loss = float(out.stdout.split("loss")[1])
    img, da, de, alb = (read_pfm(str(tmp_path / f"{k}.pfm")) for k in
                        ("image", "d_albedo", "d_emission", "albedo"))
    sd = _scene_from_record(rec)
    n = len(sd["tris"])
    assert alb.shape == (1, n, 3) and da.shape == (1, n, 3)
    # the per-triangle albedo of the scene's materials (emissive triangles 0)
    mats = np.asarray([m["color"] for m in sd["materials"]], np.float32)
    np.testing.assert_array_equal(alb[0], mats[sd["tri_material"]])
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 48, 32, 8, max_depth=4, seed=7)
    a = alb[0]
    target = sc.adjoint_forward(p, (a + np.float32(-0.2) * a).astype(np.float32), None)
    py_img = sc.adjoint_forward(p, a, None)
    loss, g = db.loss_l2(py_img, target)
    pda, pde = sc.adjoint_backward(p, g, a, sd["tri_emission"])
    np.testing.assert_allclose(img, py_img, rtol=1e-5, atol=1e-6)
    assert abs(lua_loss - loss) <= 1e-5 * abs(loss)
    np.testing.assert_allclose(da[0], pda, rtol=1e-3, atol=1e-5 * np.abs(pda).max())
    np.testing.assert_allclose(de[0], pde, rtol=1e-3, atol=1e-5 * np.abs(pde).max())
    assert np.abs(pda).max() > 0 and np.abs(pde[sd["tri_emission"].sum(1) > 0]).min() > 0


@needs_frontend
@pytest.mark.gpu
def test_script_autotune_renders_like_the_python_api(tmp_path, cuda):
    """render.make { autotune = true }: the wavefront tuned on the frame first;
    the image is the same estimator's (same random numbers)."""
    import dort_b200 as db
    from dort_b200.image import read_rgbe, rgbe_quantize
    script = tmp_path / "scene.lua"
    script.write_text(SCENE_LUA.replace("max_depth = 4,", "max_depth = 4, autotune = true,"))
    out = subprocess.run([DORT, str(script), str(tmp_path / "img.hdr")], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lua_img = read_rgbe(str(tmp_path / "img.hdr"))
    d = _python_scene()
    sc = db.scene_from_dict(d)
    p = db.render_params(d["camera"], 96, 64, 16, max_depth=4, seed=7)
    py_img = rgbe_quantize(sc.render_wavefront(p)[0])
    sc.close()
    diff = np.abs(lua_img.astype(np.float64) - py_img)
    assert float(diff.mean()) < 1e-3 * max(float(py_img.mean()), 1e-6), float(diff.mean())
