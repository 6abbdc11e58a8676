-- dort.std: small table and output helpers scene scripts use (the
-- reference's lua/dort/std.lua names: printf, clone, merge).
local std = {}

-- io.write of a string.format result
function std.printf(fmt, ...)
  return io.write(string.format(fmt, ...))
end

-- shallow copy of a table
function std.clone(t)
  local out = {}
  for k, v in pairs(t) do out[k] = v end
  return out
end

-- a new table with the keys of a and b; b wins where both have a key
function std.merge(a, b)
  local out = std.clone(a)
  for k, v in pairs(b) do out[k] = v end
  return out
end

dort.std = std
return std
