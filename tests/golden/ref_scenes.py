"""The reference's image-test scenes, restated through dort_b200.builder.

The reference checks its renderers against converged images stored in its
test/ref/*.hdr, made by its own "pt" renderer from the scenes of
test/test_box.lua, test/test_simple.lua and test/test_bsdf.lua.  This module
rebuilds those scenes (same geometry, materials, lights, cameras, in the
same builder calls) and lists, for every stored image whose scene this path
can render, the parameters that image was rendered with.  The fixture
script gen_ref_images.py reduces the stored images to the statistics the
tests compare; the GPU tests render the scenes listed here.

Not covered: the "envi" scenes (their environment map data/vogl_14.hdr is
not in the reference tree), the "beam" light scenes (a beam light is a
delta position + delta direction light that the "pt" renderer cannot see),
and the simple_*_diel / simple_*_thdi images, whose scenes are no longer in
test_simple.lua.
"""
from __future__ import annotations

import math

from dort_b200.builder import (Builder, cube, dielectric_material, disk, lambert_material,
                               look_at, mirror_material, oren_nayar_material, ortho_camera,
                               phong_material, pinhole_camera, point, rgb, rgbh, rotate_x,
                               rotate_y, scale, sphere, thin_lens_camera, translate, vector,
                               infinite_light)

PI = math.pi
CORNELL_SCALE = 0.01


def cornell_scene(geom_kind: str, surface_kind: str, light_kind: str, camera_kind: str) -> dict:
    """cornell_scene of test_box.lua:2-196."""
    s = CORNELL_SCALE
    B = Builder()
    white = lambert_material(rgb(0.5, 0.5, 0.5))
    green = lambert_material(rgb(0, 0.5, 0))
    red = lambert_material(rgb(0.5, 0, 0))
    glossy_white = phong_material(rgb(0.5), exponent=50)
    glossy_red = phong_material(rgb(0.5, 0, 0), exponent=50)
    mirror = mirror_material(rgb(1))
    glass = dielectric_material(ior_inside=1.3)

    right_box, left_box, right_wall, left_wall, floor = white, white, red, green, white
    if surface_kind == "glos":
        right_box, left_box, right_wall = glossy_white, glossy_white, glossy_red
    elif surface_kind == "delt":
        right_box, left_box, left_wall = mirror, glass, mirror
    elif surface_kind != "diff":
        raise ValueError(surface_kind)
    add_walls = {"box": True, "openbox": False}[geom_kind]

    def walls():
        m = B.mesh([point(552.8 * s, 0, 0), point(0, 0, 0), point(0, 0, 559.2 * s),
                    point(549.6 * s, 0, 559.2 * s), point(556 * s, 548.8 * s, 0),
                    point(556 * s, 548.8 * s, 559.2 * s), point(0, 548.8 * s, 559.2 * s),
                    point(0, 548.8 * s, 0)],
                   [0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7, 6, 5, 3, 6, 3, 2,
                    7, 6, 2, 7, 2, 1, 0, 3, 5, 0, 5, 4])
        B.set_material(floor)
        B.add_triangle(m, 0)
        B.add_triangle(m, 3)
        if add_walls:
            for i in (6, 9, 12, 15):
                B.add_triangle(m, i)
            B.set_material(left_wall)
            B.add_triangle(m, 18)
            B.add_triangle(m, 21)
            B.set_material(right_wall)
            B.add_triangle(m, 24)
            B.add_triangle(m, 27)
    B.block(walls)

    def left():
        B.set_material(left_box)
        B.set_transform(translate(185 * s, 82.5 * s, 169 * s) * rotate_y(-0.29)
                        * scale(165 * s / 2))
        B.add_shape(cube())
    B.block(left)

    def right():
        B.set_material(right_box)
        B.set_transform(translate(368 * s, 165 * s, 351 * s) * rotate_y(-1.27)
                        * scale(165 * s / 2, 330 * s / 2, 165 * s / 2))
        B.add_shape(cube())
    B.block(right)

    if camera_kind == "pin":
        B.set_camera(pinhole_camera(
            look_at(point(278 * s, 273 * s, -800 * s), point(278 * s, 273 * s, 0),
                    vector(0, 1, 0)) * scale(1, -1, 1), fov=0.686))
    elif camera_kind == "orth":
        B.set_camera(ortho_camera(
            800 * s, look_at(point(250 * s, 200 * s, -800 * s), point(278 * s, 273 * s, 0),
                             vector(0, 1, 0)) * scale(1, -1, 1)))
    elif camera_kind == "thin":
        B.set_camera(thin_lens_camera(
            look_at(point(278 * s, 273 * s, -800 * s), point(278 * s, 273 * s, 0),
                    vector(0, 1, 0)) * scale(1, -1, 1),
            lens_radius=50 * s, focal_distance=1200 * s, fov=0.686))
    else:
        raise ValueError(camera_kind)

    if light_kind == "area":
        def area():
            B.set_material(lambert_material(rgb(0)))
            B.set_transform(translate(0, -1 * s, 0))
            m = B.mesh([point(343 * s, 548.8 * s, 227 * s), point(343 * s, 548.8 * s, 332 * s),
                        point(213 * s, 548.8 * s, 332 * s), point(213 * s, 548.8 * s, 227 * s)],
                       [2, 1, 0, 3, 2, 0])
            for index in (0, 3):
                shape = B.triangle(m, index)
                light = B.diffuse_light(shape, rgb(100))
                B.add_light(light)
                B.add_shape(shape, light)
        B.block(area)
    elif light_kind == "sphe":
        def sph():
            B.set_transform(translate(250 * s, 400 * s, 250 * s))
            B.set_material(lambert_material(rgb(0)))
            shape = sphere(20 * s)
            light = B.diffuse_light(shape, rgb(100))
            B.add_light(light)
            B.add_shape(shape, light)
        B.block(sph)
    elif light_kind == "poin":
        B.add_light(B.point_light(point(250 * s, 400 * s, 250 * s), rgb(1) * 15e4 * s * s))
    elif light_kind == "dire":
        B.add_light(B.directional_light(vector(1, -1, 5), rgb(10)))
    elif light_kind == "infi":
        B.add_light(infinite_light(rgb(1)))
    else:
        raise ValueError(light_kind)
    return B.build_scene()


def simple_scene(geom_kind: str, surface_kind: str, light_kind: str) -> dict:
    """simple_scene of test_simple.lua:6-137 (camera "pin")."""
    B = Builder()
    B.set_material({"diff": lambert_material(rgb(0.5)),
                    "glos": phong_material(rgb(0.5), exponent=50),
                    "mirr": mirror_material(rgb(1))}[surface_kind])
    if geom_kind == "sphe":
        B.add_shape(sphere(2))
    elif geom_kind == "disk":
        B.add_shape(disk(2))
    elif geom_kind == "cube":
        def c():
            B.set_transform(rotate_y(PI / 4))
            B.set_transform(rotate_x(PI / 6))
            B.add_shape(cube())
        B.block(c)
    elif geom_kind == "disk2":
        def d1():
            B.set_transform(translate(-2, 0, 0))
            B.set_transform(rotate_y(PI / 2))
            B.set_transform(rotate_x(PI / 10))
            B.add_shape(disk(2))

        def d2():
            B.set_transform(translate(2, 0, 0))
            B.set_transform(rotate_y(PI / 2))
            B.set_transform(rotate_x(-PI / 10))
            B.add_shape(disk(2))
        B.block(d1)
        B.block(d2)
    else:
        raise ValueError(geom_kind)

    def area_disk(radiance):
        def body():
            B.set_transform(look_at(point(0, 0, -6), point(0, 0, 0), vector(0, 1, 0)))
            shape = disk(1)
            light = B.diffuse_light(shape, rgb(radiance))
            B.add_light(light)
            B.add_shape(shape, light)
        B.block(body)

    if light_kind == "poin_fwd":
        B.add_light(B.point_light(point(0, 0, -3), rgb(10)))
    elif light_kind == "poin_blw":
        B.add_light(B.point_light(point(0, -3, -3), rgb(10)))
    elif light_kind == "area_fwd":
        area_disk(10)
    elif light_kind == "dire_blw":
        B.add_light(B.directional_light(vector(0, 1, 1), rgb(1)))
    elif light_kind == "mixd_2":
        B.add_light(B.point_light(point(0, -3, -3), rgb(10)))
        area_disk(3)
    elif light_kind == "mixd_3":
        B.add_light(B.point_light(point(0, -3, -3), rgb(5)))
        area_disk(3)
        B.add_light(B.directional_light(vector(0, 1, 1), rgb(5)))
    else:
        raise ValueError(light_kind)
    B.set_camera(pinhole_camera(look_at(point(0, 0, -3), point(0, 0, 0), vector(0, 1, 0)),
                                fov=PI / 2))
    return B.build_scene()


BSDF_MATERIALS = {
    # name: (material, max_depth override) -- test_bsdf.lua:56-100
    "lamb": (lambda: lambert_material(rgbh(0x0366d6)), None),
    "orennayar_0.01": (lambda: oren_nayar_material(rgbh(0x2ba545), sigma=0.01), None),
    "orennayar_0.1": (lambda: oren_nayar_material(rgbh(0x2ba545), sigma=0.1), None),
    "orennayar_0.5": (lambda: oren_nayar_material(rgbh(0x2ba545), sigma=0.5), None),
    "mirror": (lambda: mirror_material(rgb(1)), 10),
    "dielectric_1.5": (lambda: dielectric_material(ior_inside=1.5, ior_outside=1), 10),
    "dielectric_3": (lambda: dielectric_material(ior_inside=3, ior_outside=1), 10),
    "dielectric_inv1.5": (lambda: dielectric_material(ior_inside=1, ior_outside=1.5), 10),
    "phong_50": (lambda: phong_material(rgbh(0xc6830d), exponent=50), None),
    "phong_10": (lambda: phong_material(rgbh(0xc6830d), exponent=10), None),
    "phong_200": (lambda: phong_material(rgbh(0xc6830d), exponent=200), None),
}


def bsdf_scene(tested) -> dict:
    """test_scene of test_bsdf.lua:1-54."""
    B = Builder()

    def ground():
        B.set_transform(rotate_x(PI / 2))
        B.set_material(lambert_material(rgb(0.5)))
        B.add_shape(disk(5))
    B.block(ground)

    def ball():
        B.set_material(tested)
        B.set_transform(translate(-1.5, 1, 0))
        B.add_shape(sphere(1))
    B.block(ball)

    def box():
        B.set_material(tested)
        B.set_transform(translate(1.5, 1, 0))
        B.add_shape(cube())
    B.block(box)

    B.set_material(lambert_material(rgb(0)))
    B.add_light(B.point_light(point(0, 5, -3), rgb(20)))

    def lamp1():
        B.set_transform(look_at(point(-5, 5, -3), point(-1.5, 1, 0), vector(0, 1, 0)))
        B.add_diffuse_light(disk(2), rgb(2))
    B.block(lamp1)

    def lamp2():
        B.set_transform(look_at(point(5, 5, -3), point(1.5, 1, 0), vector(0, 1, 0)))
        B.add_diffuse_light(disk(4), rgb(0.7))
    B.block(lamp2)

    B.set_camera(pinhole_camera(look_at(point(0, 4, -15), point(0, 1, 1), vector(0, -1, 0)),
                                fov=PI / 6))
    return B.build_scene()


# Each case: scene kind and arguments, resolution, the reference image's
# iterations (ref_spp), render parameters, and the `variation` its test
# compares with (test.lua:101-113: 8 unless the test sets it; test_simple.lua
# sets 1 for "pt").


def _cornell_cases():
    # test_box.lua:198-330: the scene list; each scene's reference image at
    # depths min..max (plain name) and, for some, one image per single depth
    # (_d<k>); reference iterations 500 x (1 diffuse, 4 glossy, 8 delta)
    scenes = [
        ("box", "diff", "area", "pin"), ("box", "glos", "area", "pin"),
        ("box", "delt", "area", "pin"),
        ("box", "diff", "sphe", "pin"), ("box", "glos", "sphe", "pin"),
        ("box", "delt", "sphe", "pin"),
        ("box", "diff", "poin", "pin"), ("box", "glos", "poin", "pin"),
        ("box", "delt", "poin", "pin"),
        ("box", "diff", "dire", "pin"), ("box", "glos", "dire", "pin"),
        ("box", "delt", "dire", "pin"),
        ("openbox", "diff", "infi", "pin"), ("openbox", "glos", "infi", "pin"),
        ("openbox", "delt", "infi", "pin"),
        ("box", "diff", "area", "orth"), ("box", "diff", "area", "thin"),
    ]
    cases = []
    for geom, surf, light, cam in scenes:
        min_depth = 1 if light == "poin" else 0
        ref_iter = {"diff": 1, "glos": 4, "delt": 8}[surf]
        base = f"{geom}_{surf}_{light}_{cam}"
        spec = dict(kind="cornell", args=(geom, surf, light, cam), width=512, height=512,
                    ref_spp=500 * ref_iter, sample_all_lights=False, variation=8.0)
        cases.append(dict(spec, name=base, min_depth=min_depth, max_depth=3))
        for d in range(min_depth, 4):
            cases.append(dict(spec, name=f"{base}_d{d}", min_depth=d, max_depth=d))
    return cases


def _simple_cases():
    # test_simple.lua:171-230: reference iterations 100, sample_all_lights,
    # depth 1..2; mirror surfaces skip delta lights and the two-disk scene
    cases = []
    for geom in ("sphe", "disk", "cube", "disk2"):
        for surf in ("diff", "glos", "mirr"):
            for light in ("poin_fwd", "poin_blw", "area_fwd", "dire_blw", "mixd_2", "mixd_3"):
                delta_light = light != "area_fwd"
                if surf == "mirr" and (delta_light or geom == "disk2"):
                    continue
                cases.append(dict(kind="simple", args=(geom, surf, light),
                                  name=f"simple_{geom}_{surf}_{light}_pin", width=512,
                                  height=512, ref_spp=100, sample_all_lights=True,
                                  min_depth=1, max_depth=2, variation=1.0))
    return cases


def _bsdf_cases():
    # test_bsdf.lua:102-150: 512 x 338, reference iterations 512,
    # sample_all_lights, depth 1..2 (1..10 for delta materials)
    return [dict(kind="bsdf", args=(name,), name=f"bsdf_{name}", width=512, height=338,
                 ref_spp=512, sample_all_lights=True, min_depth=1,
                 max_depth=md if md else 2, variation=8.0)
            for name, (_, md) in BSDF_MATERIALS.items()]


CASES = _cornell_cases() + _simple_cases() + _bsdf_cases()


def case_by_name(name: str) -> dict:
    """A case of CASES by name; "<name>@square" is the same case rendered
    square (width x width), for renderers that need a square film."""
    base, _, variant = name.partition("@")
    case = next(c for c in CASES if c["name"] == base)
    if variant == "square":
        return dict(case, name=name, height=case["width"])
    return case


def build(case: dict) -> dict:
    if case["kind"] == "cornell":
        return cornell_scene(*case["args"])
    if case["kind"] == "simple":
        return simple_scene(*case["args"])
    return bsdf_scene(BSDF_MATERIALS[case["args"][0]][0]())
