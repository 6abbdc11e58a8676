-- Runs scene-test scripts written for the reference renderer (test_box.lua,
-- test_simple.lua, test_bsdf.lua of its test directory) through this
-- front-end in record mode (DORT_LUA_RECORD with "%d"): every scene the
-- scripts define is flattened and written out, nothing is rendered.  Prints
-- one line per test: "<scene number> <test name>".
--   dort record_reference_tests.lua <test dir> <script name>...
local args = dort.env.get_argv()

-- images the scripts read but the tree lacks (an environment map) are
-- replaced by a 2 x 1 grey image, so the other scenes can still be recorded
local read = dort.image.read
local stub = os.tmpname()
do
  local f = io.open(stub, "wb")
  f:write("#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 1 +X 2\n")
  f:write(string.char(128, 128, 128, 129, 128, 128, 128, 129))
  f:close()
end
dort.image.read = function(path, params)
  local hdr = params and params.hdr
  local ok, img = pcall(read, path, { hdr = hdr })
  if ok then return img end
  return read(stub, { hdr = hdr })
end
local dir = args[1]
local scene_ids, next_id = {}, 0
local t = {}
function t:test(def)
  if scene_ids[def.scene] == nil then
    scene_ids[def.scene] = next_id
    next_id = next_id + 1
  end
  print(scene_ids[def.scene], def.name)
end
for i = 2, #args do
  local define_tests = dofile(dir .. "/" .. args[i] .. ".lua")
  define_tests(t)
end
