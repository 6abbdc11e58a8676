// `dort`: runs a scene script with the reference renderer's command line
// (src/dort/main.cpp: dort [options] [--] <program.lua> [program args]) and
// Lua environment (main.cpp:142-220: the standard libraries, the `dort`
// global with its modules, require of "dort/dsl" and "dort/std"), rendering
// through the B200 library.  Thread and statistics options are accepted and
// have no effect (the renderer runs on the GPU and keeps no statistics).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "frontend.h"

// Lua modules of the front-end, embedded at build time (lua_sources.cpp,
// generated from dort_b200/frontend/lua/dort/*.lua).
struct EmbeddedLua { const char* name; const char* source; };
extern const EmbeddedLua kEmbeddedLua[];

namespace {

const char* kShortUsage =
    "Usage: dort [options] [--] <program.lua> [program args]\n"
    "  Options: -t <count> | -s <word> | -S <word> | -h | -v\n";

const char* find_embedded(const std::string& name) {
  for(const EmbeddedLua* e = kEmbeddedLua; e->name; ++e) {
    if(name == e->name) { return e->source; }
  }
  return nullptr;
}

// package.searchers entry: "dort" is the global table; "dort/x" / "dort.x"
// are the embedded modules
int builtin_searcher(lua_State* l) {
  std::string name = luaL_checkstring(l, 1);
  if(name == "dort") {
    lua_pushcfunction(l, [](lua_State* ls) -> int {
      lua_getglobal(ls, "dort");
      return 1;
    });
    return 1;
  }
  for(char& c : name) { if(c == '.') { c = '/'; } }
  const char* src = find_embedded(name);
  if(!src) {
    lua_pushfstring(l, "\n\tno built-in module '%s'", name.c_str());
    return 1;
  }
  if(luaL_loadbufferx(l, src, std::strlen(src), name.c_str(), "t") != LUA_OK) {
    return lua_error(l);
  }
  return 1;
}

void run_embedded(lua_State* l, const char* name) {
  const char* src = find_embedded(name);
  if(!src || luaL_loadbufferx(l, src, std::strlen(src), name, "t") != LUA_OK) {
    lua_error(l);
  }
  lua_call(l, 0, 0);
}

int traceback(lua_State* l) {
  const char* msg = lua_tostring(l, 1);
  if(msg) { luaL_traceback(l, l, msg, 1); }
  return 1;
}

int main_lua(lua_State* l, const char* script) {
  luaL_openlibs(l);

  // built-in modules are searched first, then Lua's own (files)
  lua_getglobal(l, "package");
  lua_getfield(l, -1, "searchers");
  lua_Integer n = luaL_len(l, -1);
  for(lua_Integer i = n; i >= 1; --i) {
    lua_rawgeti(l, -1, i);
    lua_rawseti(l, -2, i + 1);
  }
  lua_pushcfunction(l, builtin_searcher);
  lua_rawseti(l, -2, 1);
  lua_pop(l, 2);

  struct { const char* name; lua_CFunction open; } subs[] = {
      {"builder", dortlua::open_builder}, {"camera", dortlua::open_camera},
      {"chrono", dortlua::open_chrono}, {"env", dortlua::open_env},
      {"filter", dortlua::open_filter}, {"geometry", dortlua::open_geometry},
      {"image", dortlua::open_image}, {"light", dortlua::open_light},
      {"material", dortlua::open_material}, {"math", dortlua::open_math},
      {"render", dortlua::open_render}, {"sampler", dortlua::open_sampler},
      {"shape", dortlua::open_shape}, {"spectrum", dortlua::open_spectrum},
      {"stats", dortlua::open_stats}, {"texture", dortlua::open_texture}};
  lua_newtable(l);
  for(const auto& s : subs) {
    std::string global = std::string("dort.") + s.name;
    luaL_requiref(l, global.c_str(), s.open, 0);
    lua_setfield(l, -2, s.name);
  }
  lua_setglobal(l, "dort");
  run_embedded(l, "dort/builder_ext");
  run_embedded(l, "dort/geometry_ext");
  run_embedded(l, "dort/std");

  lua_pushcfunction(l, traceback);
  if(luaL_loadfile(l, script) != LUA_OK) {
    std::fprintf(stderr, "Load error: %s\n", lua_tostring(l, -1));
    return 1;
  }
  if(lua_pcall(l, 0, 0, -2) != LUA_OK) {
    std::fprintf(stderr, "Runtime error: %s\n", lua_tostring(l, -1));
    return 1;
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::vector<std::string> script_argv;
  const char* script = nullptr;
  bool ok = true;
  int i = 1;
  while(i < argc) {
    std::string a = argv[i];
    if(a == "--") { ++i; break; }
    if(a == "-t" || a == "--threads" || a == "-s" || a == "--enable-stats" || a == "-S" ||
       a == "--disable-stats") {
      if(i + 1 >= argc) { ok = false; break; }
      i += 2;
    } else if(a == "-h" || a == "-?" || a == "--help") {
      std::fprintf(stdout, "%s", kShortUsage);
      return 0;
    } else if(a == "-v" || a == "--version") {
      std::fprintf(stdout, "dort (B200 path tracer, ABI %d)\n", dort_gpu_abi_version());
      return 0;
    } else if(!a.empty() && a[0] == '-') {
      ok = false;
      break;
    } else {
      break;
    }
  }
  if(i < argc) { script = argv[i++]; } else { ok = false; }
  for(; i < argc; ++i) { script_argv.push_back(argv[i]); }
  if(!ok) {
    std::fprintf(stderr, "%s", kShortUsage);
    return 3;
  }
  dortlua::set_argv(script_argv);
  lua_State* l = luaL_newstate();
  int rc = main_lua(l, script);
  lua_close(l);
  return rc;
}
