-- Transforms around a point (the reference's lua/dort/geometry_ext.lua
-- names): move origin to zero, apply, move back.
local g = dort.geometry

local function around(t, origin)
  local x, y, z = origin:x(), origin:y(), origin:z()
  return g.translate(x, y, z) * t * g.translate(-x, -y, -z)
end

function g.rotate_x_around(angle, origin) return around(g.rotate_x(angle), origin) end
function g.rotate_y_around(angle, origin) return around(g.rotate_y(angle), origin) end
function g.rotate_z_around(angle, origin) return around(g.rotate_z(angle), origin) end

function g.scale_around(s, origin)
  if type(s) == "number" then
    return around(g.scale(s), origin)
  end
  return around(g.scale(s:x(), s:y(), s:z()), origin)
end
