-- The scene-description DSL (`local _ENV = require "dort/dsl"`): the names
-- of the reference's lua/dort/dsl.lua, over one current builder.  Functions
-- that place things (lights, meshes) put the builder's transform in front of
-- their own.
local dsl = {}
for k, v in pairs(_G) do dsl[k] = v end
for k, v in pairs(dort.math) do dsl[k] = v end

local b = dort.builder
local B = nil

local function current()
  if not B then error("no scene is being defined (use define_scene)", 3) end
  return B
end

local function placed(transform)
  local t = b.get_transform(current())
  if transform then return t * transform end
  return t
end

function dsl.get_builder() return B end
function dsl.get_transform() return b.get_transform(current()) end

function dsl.define_scene(callback)
  local saved = B
  B = b.make()
  local ok, err = pcall(callback, B)
  if not ok then B = saved; error(err, 0) end
  local scene = b.build_scene(B)
  B = saved
  return scene
end

function dsl.block(callback) return b.block(current(), callback) end
function dsl.frame(callback) return b.frame(current(), callback) end
function dsl.transform(t) b.set_transform(current(), t) end
function dsl.material(m) b.set_material(current(), m) end
function dsl.camera(c) b.set_camera(current(), c) end
function dsl.option(name, ...) b.set_option(current(), name, ...) end

function dsl.add_shape(shape, ...) b.add_shape(current(), shape, ...) end
function dsl.add_primitive(prim) b.add_primitive(current(), prim) end
function dsl.add_triangle(mesh, index) b.add_triangle(current(), mesh, index) end
function dsl.add_light(light) b.add_light(current(), light) end
function dsl.add_read_ply_mesh(file) b.add_read_ply_mesh(current(), file) end
function dsl.add_read_ply_mesh_as_bvh(file) b.add_read_ply_mesh_as_bvh(current(), file) end
function dsl.add_ply_mesh(mesh) b.add_ply_mesh(current(), mesh) end
function dsl.add_ply_mesh_as_bvh(mesh) b.add_ply_mesh_as_bvh(current(), mesh) end
function dsl.add_voxel_grid(params) b.add_voxel_grid(current(), params) end
function dsl.add_diffuse_light(params)
  params.transform = placed(params.transform)
  b.add_diffuse_light(current(), params)
end

-- render(scene, params): renders synchronously; params.hdr selects the float
-- image (default: 8-bit)
function dsl.render(scene, params)
  local hdr = params.hdr
  params.hdr = nil
  local job = dort.render.make(scene, params)
  dort.render.render_sync(job)
  return dort.render.get_image(job, { hdr = hdr })
end

dsl.pinhole_camera = dort.camera.make_pinhole
dsl.ortho_camera = dort.camera.make_ortho
dsl.thin_lens_camera = dort.camera.make_thin_lens

dsl.box_filter = dort.filter.make_box
dsl.triangle_filter = dort.filter.make_triangle
dsl.gaussian_filter = dort.filter.make_gaussian
dsl.mitchell_filter = dort.filter.make_mitchell
dsl.lanczos_sinc_filter = dort.filter.make_lanczos_sinc

local g = dort.geometry
for _, name in ipairs({"vector", "point", "identity", "inverse", "translate", "scale",
    "rotate_x", "rotate_y", "rotate_z", "rotate_x_around", "rotate_y_around",
    "rotate_z_around", "look_at", "stretch", "vec3i", "vec2", "boxi"}) do
  dsl[name] = g[name]
end

dsl.read_image = dort.image.read
dsl.write_png_image = dort.image.write_png
dsl.write_rgbe_image = dort.image.write_rgbe
dsl.tonemap_srgb = dort.image.tonemap_srgb
dsl.tonemap_gamma = dort.image.tonemap_gamma

local function placed_light(make)
  return function(params)
    params.transform = placed(params.transform)
    return make(params)
  end
end
dsl.point_light = placed_light(dort.light.make_point)
dsl.diffuse_light = placed_light(dort.light.make_diffuse)
dsl.directional_light = placed_light(dort.light.make_directional)
dsl.environment_light = placed_light(dort.light.make_environment)
dsl.beam_light = placed_light(dort.light.make_beam)
dsl.infinite_light = dort.light.make_infinite

dsl.lambert_material = dort.material.make_lambert
dsl.oren_nayar_material = dort.material.make_oren_nayar
dsl.mirror_material = dort.material.make_mirror
dsl.dielectric_material = dort.material.make_dielectric
dsl.rough_dielectric_material = dort.material.make_rough_dielectric
dsl.phong_material = dort.material.make_phong
dsl.bump_material = dort.material.make_bump

dsl.random_sampler = dort.sampler.make_random
dsl.stratified_sampler = dort.sampler.make_stratified

dsl.sphere = dort.shape.make_sphere
dsl.disk = dort.shape.make_disk
dsl.cylinder = dort.shape.make_cylinder
dsl.cube = dort.shape.make_cube
dsl.polygon = dort.shape.make_polygon
dsl.read_ply_mesh = dort.shape.read_ply_mesh

function dsl.mesh(params)
  if not params.transform then params.transform = b.get_transform(current()) end
  return dort.shape.make_mesh(params)
end

function dsl.triangle(mesh, index) return b.make_triangle(current(), mesh, index) end

dsl.rgb = dort.spectrum.rgb
dsl.rgbh = dort.spectrum.rgbh

dsl.reset_stats = dort.stats.reset
dsl.write_and_reset_stats = dort.stats.write_and_reset

local tex = dort.texture
dsl.compose_texture = tex.compose
dsl.const_texture = tex.make_const_geom
dsl.const_texture_1d = tex.make_const_1d
dsl.const_texture_2d = tex.make_const_2d
dsl.const_texture_3d = tex.make_const_3d
dsl.identity_texture_1d = tex.make_identity_1d
dsl.identity_texture_2d = tex.make_identity_2d
dsl.identity_texture_3d = tex.make_identity_3d
dsl.lerp_texture = tex.make_lerp
dsl.checkerboard_texture_1d = tex.make_checkerboard_1d
dsl.checkerboard_texture_2d = tex.make_checkerboard_2d
dsl.checkerboard_texture_3d = tex.make_checkerboard_3d
dsl.image_texture = tex.make_image
dsl.gain_texture = tex.make_gain
dsl.bias_texture = tex.make_bias
dsl.uv_texture_map = tex.make_map_uv
dsl.xy_texture_map = tex.make_map_xy
dsl.spherical_texture_map = tex.make_map_spherical
dsl.cylindrical_texture_map = tex.make_map_cylindrical
dsl.xyz_texture_map = tex.make_map_xyz
dsl.grayscale_color_map = tex.make_color_map_grayscale
dsl.lerp_color_map = tex.make_color_map_lerp
dsl.spline_color_map = tex.make_color_map_spline
dsl.render_texture_2d = tex.render_2d
for _, d in ipairs({"1d", "2d", "3d"}) do
  for _, of in ipairs({"", "_of_2d", "_of_3d"}) do
    dsl["value_noise_texture_" .. d .. of] = tex["make_value_noise_" .. d .. of]
  end
end

dort.dsl = dsl
return dsl
