-- Builder helpers defined in Lua (the reference's lua/dort/builder_ext.lua
-- names: block, frame, add_diffuse_light).
local b = dort.builder

-- runs callback(B) with the builder state saved and restored around it
function b.block(B, callback)
  b.push_state(B)
  local result = callback(B)
  b.pop_state(B)
  return result
end

-- collects what callback(B) adds into one primitive (a frame) and returns it
function b.frame(B, callback)
  b.push_frame(B)
  callback(B)
  return b.pop_frame(B)
end

-- a diffuse light with params (shape, radiance, transform) and its shape as a
-- primitive with a black Lambert material; as in the reference, the shape is
-- added after set_transform(params.transform), which composes with the
-- builder's current transform
function b.add_diffuse_light(B, params)
  local shape, transform = params.shape, params.transform
  local light = dort.light.make_diffuse(params)
  b.block(B, function()
    b.set_transform(B, transform)
    b.set_material(B, dort.material.make_lambert { albedo = dort.spectrum.rgb(0) })
    b.add_shape(B, shape, light)
  end)
  b.add_light(B, light)
end
