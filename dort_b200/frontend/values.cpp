// Values of the Lua front-end: vectors / points / normals, transforms,
// spectra, small integer vectors and rectangles, parameter tables, and the
// dort.geometry, dort.spectrum and dort.math modules (the reference's
// lua_geometry.cpp, lua_spectrum.cpp, lua_math.cpp, lua_params.cpp).
#include <cmath>
#include <cstring>
#include <random>

#include "frontend.h"

namespace dortlua {

// ---- matrices ---------------------------------------------------------------------

Mat4 Mat4::identity() {
  Mat4 r;
  for(int i = 0; i < 4; ++i) {
    for(int j = 0; j < 4; ++j) { r.m[i][j] = i == j ? 1.0 : 0.0; }
  }
  return r;
}

Mat4 Mat4::operator*(const Mat4& o) const {
  Mat4 r;
  for(int i = 0; i < 4; ++i) {
    for(int j = 0; j < 4; ++j) {
      double s = 0.0;
      for(int k = 0; k < 4; ++k) { s += m[i][k] * o.m[k][j]; }
      r.m[i][j] = s;
    }
  }
  return r;
}

V3 Mat4::point(V3 p) const {
  return {m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z + m[0][3],
          m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z + m[1][3],
          m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z + m[2][3]};
}

V3 Mat4::vector(V3 v) const {
  return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
          m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
          m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}

Mat4 Mat4::inverse() const {
  // Gauss-Jordan with partial pivoting
  double a[4][8];
  for(int i = 0; i < 4; ++i) {
    for(int j = 0; j < 4; ++j) { a[i][j] = m[i][j]; a[i][j + 4] = i == j ? 1.0 : 0.0; }
  }
  for(int c = 0; c < 4; ++c) {
    int piv = c;
    for(int r = c + 1; r < 4; ++r) {
      if(std::fabs(a[r][c]) > std::fabs(a[piv][c])) { piv = r; }
    }
    if(piv != c) { for(int j = 0; j < 8; ++j) { std::swap(a[c][j], a[piv][j]); } }
    double d = a[c][c];
    if(d == 0.0) { return identity(); }
    for(int j = 0; j < 8; ++j) { a[c][j] /= d; }
    for(int r = 0; r < 4; ++r) {
      if(r == c) { continue; }
      double f = a[r][c];
      for(int j = 0; j < 8; ++j) { a[r][j] -= f * a[c][j]; }
    }
  }
  Mat4 r;
  for(int i = 0; i < 4; ++i) {
    for(int j = 0; j < 4; ++j) { r.m[i][j] = a[i][j + 4]; }
  }
  return r;
}

bool Mat4::operator==(const Mat4& o) const { return std::memcmp(m, o.m, sizeof(m)) == 0; }

// ---- userdata plumbing ---------------------------------------------------------------

void register_type(lua_State* l, const char* tname, const luaL_Reg* methods, lua_CFunction gc) {
  luaL_newmetatable(l, tname);
  lua_newtable(l);   // __index
  for(const luaL_Reg* r = methods; r && r->name; ++r) {
    lua_pushcfunction(l, r->func);
    if(std::strncmp(r->name, "__", 2) == 0) {
      lua_setfield(l, -3, r->name);
    } else {
      lua_setfield(l, -2, r->name);
    }
  }
  lua_setfield(l, -2, "__index");
  if(gc) {
    lua_pushcfunction(l, gc);
    lua_setfield(l, -2, "__gc");
  }
  lua_pushstring(l, tname);
  lua_setfield(l, -2, "__name");
  lua_pop(l, 1);
}

static const char* kind_tname(VecKind k) {
  return k == KIND_VECTOR ? VEC_T : (k == KIND_POINT ? PNT_T : NRM_T);
}

bool test_vec3(lua_State* l, int idx, VecKind kind) {
  return luaL_testudata(l, idx, kind_tname(kind)) != nullptr;
}

V3 check_vec3(lua_State* l, int idx, VecKind kind) {
  return *static_cast<V3*>(luaL_checkudata(l, idx, kind_tname(kind)));
}

void push_vec3(lua_State* l, VecKind kind, V3 v) { push_value(l, kind_tname(kind), v); }

Transform check_transform(lua_State* l, int idx) {
  return *static_cast<Transform*>(luaL_checkudata(l, idx, XF_T));
}

void push_transform(lua_State* l, const Transform& t) { push_value(l, XF_T, t); }

Spectrum check_spectrum(lua_State* l, int idx) {
  if(lua_type(l, idx) == LUA_TNUMBER) {
    double x = lua_tonumber(l, idx);
    return {x, x, x};
  }
  return *static_cast<Spectrum*>(luaL_checkudata(l, idx, SPEC_T));
}

void push_spectrum(lua_State* l, Spectrum s) { push_value(l, SPEC_T, s); }

// ---- parameter tables ------------------------------------------------------------------

int params_index(lua_State* l, int idx) {
  if(lua_isnoneornil(l, idx)) {
    lua_newtable(l);
    lua_replace(l, idx);
  }
  luaL_checktype(l, idx, LUA_TTABLE);
  return lua_absindex(l, idx);
}

bool param_take(lua_State* l, int p, const char* name) {
  lua_getfield(l, p, name);
  if(lua_isnil(l, -1)) {
    lua_pop(l, 1);
    return false;
  }
  lua_pushnil(l);
  lua_setfield(l, p, name);
  return true;
}

double param_number(lua_State* l, int p, const char* name) {
  if(!param_take(l, p, name)) { luaL_error(l, "Missing parameter '%s'", name); }
  if(!lua_isnumber(l, -1)) { luaL_error(l, "Parameter '%s' must be a number", name); }
  double v = lua_tonumber(l, -1);
  lua_pop(l, 1);
  return v;
}

double param_number_opt(lua_State* l, int p, const char* name, double def) {
  lua_getfield(l, p, name);
  bool present = !lua_isnil(l, -1);
  lua_pop(l, 1);
  return present ? param_number(l, p, name) : def;
}

uint32_t param_uint_opt(lua_State* l, int p, const char* name, uint32_t def) {
  double v = param_number_opt(l, p, name, double(def));
  if(!(v >= 0.0) || v > 4294967295.0 || v != std::floor(v)) {
    luaL_error(l, "Parameter '%s' must be a non-negative integer", name);
  }
  return uint32_t(v);
}

bool param_bool_opt(lua_State* l, int p, const char* name, bool def) {
  if(!param_take(l, p, name)) { return def; }
  bool v = lua_toboolean(l, -1);
  lua_pop(l, 1);
  return v;
}

std::string param_string_opt(lua_State* l, int p, const char* name, const std::string& def) {
  if(!param_take(l, p, name)) { return def; }
  if(!lua_isstring(l, -1)) { luaL_error(l, "Parameter '%s' must be a string", name); }
  std::string v = lua_tostring(l, -1);
  lua_pop(l, 1);
  return v;
}

Spectrum param_spectrum(lua_State* l, int p, const char* name) {
  if(!param_take(l, p, name)) { luaL_error(l, "Missing parameter '%s'", name); }
  if(lua_type(l, -1) != LUA_TNUMBER && !luaL_testudata(l, -1, SPEC_T)) {
    luaL_error(l, "Parameter '%s' must be a spectrum or a number (textures other than "
                  "constants are not supported)", name);
  }
  Spectrum s = check_spectrum(l, -1);
  lua_pop(l, 1);
  return s;
}

Spectrum param_spectrum_opt(lua_State* l, int p, const char* name, Spectrum def) {
  lua_getfield(l, p, name);
  bool present = !lua_isnil(l, -1);
  lua_pop(l, 1);
  return present ? param_spectrum(l, p, name) : def;
}

Transform param_transform(lua_State* l, int p, const char* name) {
  if(!param_take(l, p, name)) { luaL_error(l, "Missing parameter '%s'", name); }
  Transform t = check_transform(l, -1);
  lua_pop(l, 1);
  return t;
}

Transform param_transform_opt(lua_State* l, int p, const char* name, const Transform& def) {
  lua_getfield(l, p, name);
  bool present = !lua_isnil(l, -1);
  lua_pop(l, 1);
  return present ? param_transform(l, p, name) : def;
}

V3 param_vec3(lua_State* l, int p, const char* name, VecKind kind) {
  if(!param_take(l, p, name)) { luaL_error(l, "Missing parameter '%s'", name); }
  V3 v = check_vec3(l, -1, kind);
  lua_pop(l, 1);
  return v;
}

void params_check_unused(lua_State* l, int p) {
  lua_pushnil(l);
  if(lua_next(l, p)) {
    const char* key = lua_tostring(l, -2);
    luaL_error(l, "Unused parameter '%s'", key ? key : "?");
  }
}

// ---- dort.geometry -------------------------------------------------------------------

static int vec_kind_of(lua_State* l, int idx) {
  for(int k = 0; k < 3; ++k) {
    if(test_vec3(l, idx, VecKind(k))) { return k; }
  }
  return -1;
}

static V3 any_vec3(lua_State* l, int idx) {
  int k = vec_kind_of(l, idx);
  if(k < 0) { luaL_argerror(l, idx, "expected a vector, point or normal"); }
  return check_vec3(l, idx, VecKind(k));
}

template<VecKind K>
static int vec_make(lua_State* l) {
  if(lua_gettop(l) == 1) {
    push_vec3(l, K, any_vec3(l, 1));
  } else {
    push_vec3(l, K, {luaL_checknumber(l, 1), luaL_checknumber(l, 2), luaL_checknumber(l, 3)});
  }
  return 1;
}

static int vec_x(lua_State* l) { lua_pushnumber(l, any_vec3(l, 1).x); return 1; }
static int vec_y(lua_State* l) { lua_pushnumber(l, any_vec3(l, 1).y); return 1; }
static int vec_z(lua_State* l) { lua_pushnumber(l, any_vec3(l, 1).z); return 1; }

static int vec_length(lua_State* l) {
  V3 v = any_vec3(l, 1);
  lua_pushnumber(l, std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
  return 1;
}

static int vec_tostring(lua_State* l) {
  int k = vec_kind_of(l, 1);
  V3 v = any_vec3(l, 1);
  const char* n = k == KIND_VECTOR ? "vector" : (k == KIND_POINT ? "point" : "normal");
  lua_pushfstring(l, "%s(%f, %f, %f)", n, v.x, v.y, v.z);
  return 1;
}

// lua_geometry.cpp:157-220: the combinations the reference allows
static int geo_add(lua_State* l) {
  int a = vec_kind_of(l, 1), b = vec_kind_of(l, 2);
  if(a < 0 || b < 0) { return luaL_error(l, "Wrong combination of arguments to +"); }
  V3 x = any_vec3(l, 1), y = any_vec3(l, 2);
  V3 r{x.x + y.x, x.y + y.y, x.z + y.z};
  if(a == KIND_POINT || b == KIND_POINT) {
    if(a == KIND_NORMAL || b == KIND_NORMAL) { return luaL_error(l, "Wrong combination of arguments to +"); }
    push_vec3(l, KIND_POINT, r);
  } else if(a == b) {
    push_vec3(l, VecKind(a), r);
  } else {
    return luaL_error(l, "Wrong combination of arguments to +");
  }
  return 1;
}

static int geo_sub(lua_State* l) {
  int a = vec_kind_of(l, 1), b = vec_kind_of(l, 2);
  if(a < 0 || b < 0) { return luaL_error(l, "Wrong combination of arguments to -"); }
  V3 x = any_vec3(l, 1), y = any_vec3(l, 2);
  V3 r{x.x - y.x, x.y - y.y, x.z - y.z};
  if(a == KIND_POINT && b == KIND_VECTOR) {
    push_vec3(l, KIND_POINT, r);
  } else if(a == KIND_POINT && b == KIND_POINT) {
    push_vec3(l, KIND_VECTOR, r);
  } else if(a == b) {
    push_vec3(l, VecKind(a), r);
  } else {
    return luaL_error(l, "Wrong combination of arguments to -");
  }
  return 1;
}

static int geo_mul(lua_State* l) {
  int a = vec_kind_of(l, 1);
  if(a < 0) { return luaL_error(l, "Wrong combination of arguments to *"); }
  V3 x = any_vec3(l, 1);
  double s = luaL_checknumber(l, 2);
  push_vec3(l, VecKind(a), {x.x * s, x.y * s, x.z * s});
  return 1;
}

static int geo_eq(lua_State* l) {
  int a = vec_kind_of(l, 1), b = vec_kind_of(l, 2);
  bool eq = a >= 0 && a == b;
  if(eq) {
    V3 x = any_vec3(l, 1), y = any_vec3(l, 2);
    eq = x.x == y.x && x.y == y.y && x.z == y.z;
  }
  lua_pushboolean(l, eq);
  return 1;
}

static int geo_cross(lua_State* l) {
  V3 a = any_vec3(l, 1), b = any_vec3(l, 2);
  push_vec3(l, KIND_VECTOR, {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x});
  return 1;
}

static Transform make_transform(const Mat4& m) { return {m, m.inverse()}; }

static int xf_identity(lua_State* l) { push_transform(l, Transform::identity()); return 1; }

static int xf_translate(lua_State* l) {
  V3 d = lua_gettop(l) == 1 ? check_vec3(l, 1, KIND_VECTOR)
                            : V3{luaL_checknumber(l, 1), luaL_checknumber(l, 2), luaL_checknumber(l, 3)};
  Mat4 m = Mat4::identity();
  m.m[0][3] = d.x; m.m[1][3] = d.y; m.m[2][3] = d.z;
  push_transform(l, make_transform(m));
  return 1;
}

static int xf_scale(lua_State* l) {
  double x, y, z;
  if(lua_gettop(l) == 1) {
    x = y = z = luaL_checknumber(l, 1);
  } else {
    x = luaL_checknumber(l, 1); y = luaL_checknumber(l, 2); z = luaL_checknumber(l, 3);
  }
  Mat4 m = Mat4::identity();
  m.m[0][0] = x; m.m[1][1] = y; m.m[2][2] = z;
  push_transform(l, make_transform(m));
  return 1;
}

// transform.cpp:93-127: right-handed rotations about the axes
static Transform rotation(int axis, double angle) {
  double c = std::cos(angle), s = std::sin(angle);
  int i = axis == 0 ? 1 : (axis == 1 ? 2 : 0);
  int j = axis == 0 ? 2 : (axis == 1 ? 0 : 1);
  Mat4 m = Mat4::identity();
  m.m[i][i] = c; m.m[i][j] = -s; m.m[j][i] = s; m.m[j][j] = c;
  return make_transform(m);
}
static int xf_rotate_x(lua_State* l) { push_transform(l, rotation(0, luaL_checknumber(l, 1))); return 1; }
static int xf_rotate_y(lua_State* l) { push_transform(l, rotation(1, luaL_checknumber(l, 1))); return 1; }
static int xf_rotate_z(lua_State* l) { push_transform(l, rotation(2, luaL_checknumber(l, 1))); return 1; }

static V3 normalized(V3 v) {
  double n = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  return {v.x / n, v.y / n, v.z / n};
}
static V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// transform.cpp:146-165: columns right = normalize(up x dir), up' = dir x
// right, dir; origin at eye
static int xf_look_at(lua_State* l) {
  V3 eye = check_vec3(l, 1, KIND_POINT), look = check_vec3(l, 2, KIND_POINT);
  V3 up = check_vec3(l, 3, KIND_VECTOR);
  V3 dir = normalized({look.x - eye.x, look.y - eye.y, look.z - eye.z});
  V3 right = normalized(cross3(normalized(up), dir));
  V3 u = cross3(dir, right);
  Mat4 m = Mat4::identity();
  const V3 cols[4] = {right, u, dir, eye};
  for(int c = 0; c < 4; ++c) {
    m.m[0][c] = cols[c].x; m.m[1][c] = cols[c].y; m.m[2][c] = cols[c].z;
  }
  push_transform(l, make_transform(m));
  return 1;
}

// lua_geometry.cpp:454-462: (-1,-1,-1) -> p1, (1,1,1) -> p2
static int xf_stretch(lua_State* l) {
  V3 a = check_vec3(l, 1, KIND_POINT), b = check_vec3(l, 2, KIND_POINT);
  Mat4 m = Mat4::identity();
  m.m[0][0] = 0.5 * (b.x - a.x); m.m[1][1] = 0.5 * (b.y - a.y); m.m[2][2] = 0.5 * (b.z - a.z);
  m.m[0][3] = 0.5 * (a.x + b.x); m.m[1][3] = 0.5 * (a.y + b.y); m.m[2][3] = 0.5 * (a.z + b.z);
  push_transform(l, make_transform(m));
  return 1;
}

static int xf_inverse(lua_State* l) {
  Transform t = check_transform(l, 1);
  push_transform(l, {t.inv, t.mat});
  return 1;
}

static int xf_mul(lua_State* l) {
  push_transform(l, check_transform(l, 1) * check_transform(l, 2));
  return 1;
}

static int xf_eq(lua_State* l) {
  bool eq = luaL_testudata(l, 1, XF_T) && luaL_testudata(l, 2, XF_T) &&
            check_transform(l, 1).mat == check_transform(l, 2).mat;
  lua_pushboolean(l, eq);
  return 1;
}

// lua_geometry.cpp:503-529: apply (optionally inverse) to a point or vector
static int xf_apply(lua_State* l) {
  Transform t = check_transform(l, 1);
  int arg = 2;
  bool inv = false;
  if(lua_isboolean(l, 2)) { inv = lua_toboolean(l, 2); arg = 3; }
  const Mat4& m = inv ? t.inv : t.mat;
  if(test_vec3(l, arg, KIND_POINT)) {
    push_vec3(l, KIND_POINT, m.point(check_vec3(l, arg, KIND_POINT)));
  } else if(test_vec3(l, arg, KIND_VECTOR)) {
    push_vec3(l, KIND_VECTOR, m.vector(check_vec3(l, arg, KIND_VECTOR)));
  } else {
    return luaL_argerror(l, arg, "Expected point or vector");
  }
  return 1;
}

static int xf_apply_inv(lua_State* l) {
  lua_pushboolean(l, true);
  lua_insert(l, 2);
  return xf_apply(l);
}

static int xf_call(lua_State* l) { return xf_apply(l); }

static int xf_tostring(lua_State* l) {
  Transform t = check_transform(l, 1);
  luaL_Buffer b;
  luaL_buffinit(l, &b);
  luaL_addstring(&b, "transform(");
  for(int r = 0; r < 4; ++r) {
    char row[160];
    std::snprintf(row, sizeof(row), "%s[%g, %g, %g, %g]", r ? ", " : "", t.mat.m[r][0],
                  t.mat.m[r][1], t.mat.m[r][2], t.mat.m[r][3]);
    luaL_addstring(&b, row);
  }
  luaL_addstring(&b, ")");
  luaL_pushresult(&b);
  return 1;
}

// small integer vectors and rectangles (vec2, vec2i, vec3i, boxi, recti)
struct Vec2 { double x, y; };
struct Vec2i { int64_t x, y; };
struct Vec3i { int64_t x, y, z; };
struct Boxi { Vec3i lo, hi; };
struct Recti { Vec2i lo, hi; };

static int vec2_make(lua_State* l) {
  push_value(l, VEC2_T, Vec2{luaL_checknumber(l, 1), luaL_checknumber(l, 2)});
  return 1;
}
static int vec2i_make(lua_State* l) {
  push_value(l, VEC2I_T, Vec2i{luaL_checkinteger(l, 1), luaL_checkinteger(l, 2)});
  return 1;
}
static int vec3i_make(lua_State* l) {
  push_value(l, VEC3I_T,
             Vec3i{luaL_checkinteger(l, 1), luaL_checkinteger(l, 2), luaL_checkinteger(l, 3)});
  return 1;
}
static int boxi_make(lua_State* l) {
  Vec3i a = *static_cast<Vec3i*>(luaL_checkudata(l, 1, VEC3I_T));
  Vec3i b = *static_cast<Vec3i*>(luaL_checkudata(l, 2, VEC3I_T));
  push_value(l, BOXI_T, Boxi{a, b});
  return 1;
}
// recti(x0, y0, x1, y1) or recti(vec2i, vec2i)
static int recti_make(lua_State* l) {
  Recti r;
  if(lua_gettop(l) == 2) {
    r.lo = *static_cast<Vec2i*>(luaL_checkudata(l, 1, VEC2I_T));
    r.hi = *static_cast<Vec2i*>(luaL_checkudata(l, 2, VEC2I_T));
  } else {
    r.lo = {luaL_checkinteger(l, 1), luaL_checkinteger(l, 2)};
    r.hi = {luaL_checkinteger(l, 3), luaL_checkinteger(l, 4)};
  }
  push_value(l, RECTI_T, r);
  return 1;
}
static int v2_x(lua_State* l) {
  if(auto* v = static_cast<Vec2*>(luaL_testudata(l, 1, VEC2_T))) { lua_pushnumber(l, v->x); }
  else { lua_pushinteger(l, static_cast<Vec2i*>(luaL_checkudata(l, 1, VEC2I_T))->x); }
  return 1;
}
static int v2_y(lua_State* l) {
  if(auto* v = static_cast<Vec2*>(luaL_testudata(l, 1, VEC2_T))) { lua_pushnumber(l, v->y); }
  else { lua_pushinteger(l, static_cast<Vec2i*>(luaL_checkudata(l, 1, VEC2I_T))->y); }
  return 1;
}
static int v3i_x(lua_State* l) { lua_pushinteger(l, static_cast<Vec3i*>(luaL_checkudata(l, 1, VEC3I_T))->x); return 1; }
static int v3i_y(lua_State* l) { lua_pushinteger(l, static_cast<Vec3i*>(luaL_checkudata(l, 1, VEC3I_T))->y); return 1; }
static int v3i_z(lua_State* l) { lua_pushinteger(l, static_cast<Vec3i*>(luaL_checkudata(l, 1, VEC3I_T))->z); return 1; }

// rectangles the reference's tests pass to image functions
bool check_recti(lua_State* l, int idx, int64_t out[4]) {
  Recti* r = static_cast<Recti*>(luaL_checkudata(l, idx, RECTI_T));
  out[0] = r->lo.x; out[1] = r->lo.y; out[2] = r->hi.x; out[3] = r->hi.y;
  return true;
}

int open_geometry(lua_State* l) {
  const luaL_Reg vec_methods[] = {
      {"x", vec_x}, {"y", vec_y}, {"z", vec_z}, {"length", vec_length},
      {"__tostring", vec_tostring}, {"__add", geo_add}, {"__sub", geo_sub},
      {"__mul", geo_mul}, {"__eq", geo_eq}, {nullptr, nullptr}};
  register_type(l, VEC_T, vec_methods, nullptr);
  register_type(l, PNT_T, vec_methods, nullptr);
  register_type(l, NRM_T, vec_methods, nullptr);
  const luaL_Reg xf_methods[] = {
      {"apply", xf_apply}, {"apply_inv", xf_apply_inv}, {"__call", xf_call},
      {"__mul", xf_mul}, {"__eq", xf_eq}, {"__tostring", xf_tostring}, {nullptr, nullptr}};
  register_type(l, XF_T, xf_methods, nullptr);
  const luaL_Reg v2_methods[] = {{"x", v2_x}, {"y", v2_y}, {nullptr, nullptr}};
  register_type(l, VEC2_T, v2_methods, nullptr);
  register_type(l, VEC2I_T, v2_methods, nullptr);
  const luaL_Reg v3i_methods[] = {{"x", v3i_x}, {"y", v3i_y}, {"z", v3i_z}, {nullptr, nullptr}};
  register_type(l, VEC3I_T, v3i_methods, nullptr);
  const luaL_Reg empty[] = {{nullptr, nullptr}};
  register_type(l, BOXI_T, empty, nullptr);
  register_type(l, RECTI_T, empty, nullptr);
  const luaL_Reg funs[] = {
      {"vector", vec_make<KIND_VECTOR>}, {"point", vec_make<KIND_POINT>},
      {"normal", vec_make<KIND_NORMAL>}, {"cross", geo_cross},
      {"identity", xf_identity}, {"inverse", xf_inverse}, {"translate", xf_translate},
      {"scale", xf_scale}, {"rotate_x", xf_rotate_x}, {"rotate_y", xf_rotate_y},
      {"rotate_z", xf_rotate_z}, {"look_at", xf_look_at}, {"stretch", xf_stretch},
      {"vec3i", vec3i_make}, {"vec2i", vec2i_make}, {"vec2", vec2_make},
      {"boxi", boxi_make}, {"recti", recti_make}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- dort.spectrum ---------------------------------------------------------------

static int spec_rgb(lua_State* l) {
  if(lua_gettop(l) == 1) {
    double x = luaL_checknumber(l, 1);
    push_spectrum(l, {x, x, x});
  } else {
    push_spectrum(l, {luaL_checknumber(l, 1), luaL_checknumber(l, 2), luaL_checknumber(l, 3)});
  }
  return 1;
}

// lua_spectrum.cpp:62-101: "#rrggbb" / "rrggbb", 0xrrggbb or three 0..255 numbers
static int spec_rgbh(lua_State* l) {
  double r, g, b;
  if(lua_type(l, 1) == LUA_TSTRING) {
    const char* s = lua_tostring(l, 1);
    if(s[0] == '#') { ++s; }
    if(std::strlen(s) < 6) { return luaL_argerror(l, 1, "A hex-format color must have 6 hex-digits"); }
    uint32_t hex = 0;
    for(int i = 0; i < 6; ++i) {
      char c = s[i];
      uint32_t d;
      if(c >= '0' && c <= '9') { d = uint32_t(c - '0'); }
      else if(c >= 'a' && c <= 'f') { d = uint32_t(c - 'a' + 10); }
      else if(c >= 'A' && c <= 'F') { d = uint32_t(c - 'A' + 10); }
      else { return luaL_argerror(l, 1, "A hex-format color must have 6 hex-digits"); }
      hex = (hex << 4) | d;
    }
    r = ((hex >> 16) & 0xff) / 255.0; g = ((hex >> 8) & 0xff) / 255.0; b = (hex & 0xff) / 255.0;
  } else if(lua_gettop(l) >= 3) {
    r = luaL_checknumber(l, 1) / 255.0; g = luaL_checknumber(l, 2) / 255.0;
    b = luaL_checknumber(l, 3) / 255.0;
  } else {
    lua_Integer hex = luaL_checkinteger(l, 1);
    r = ((hex >> 16) & 0xff) / 255.0; g = ((hex >> 8) & 0xff) / 255.0; b = (hex & 0xff) / 255.0;
  }
  push_spectrum(l, {float(r), float(g), float(b)});
  return 1;
}

static Spectrum spec_bin(Spectrum a, Spectrum b, char op) {
  switch(op) {
    case '+': return {a.r + b.r, a.g + b.g, a.b + b.b};
    case '-': return {a.r - b.r, a.g - b.g, a.b - b.b};
    case '*': return {a.r * b.r, a.g * b.g, a.b * b.b};
    default: return {a.r / b.r, a.g / b.g, a.b / b.b};
  }
}
static int spec_add(lua_State* l) { push_spectrum(l, spec_bin(check_spectrum(l, 1), check_spectrum(l, 2), '+')); return 1; }
static int spec_sub(lua_State* l) { push_spectrum(l, spec_bin(check_spectrum(l, 1), check_spectrum(l, 2), '-')); return 1; }
static int spec_mul(lua_State* l) { push_spectrum(l, spec_bin(check_spectrum(l, 1), check_spectrum(l, 2), '*')); return 1; }
static int spec_div(lua_State* l) { push_spectrum(l, spec_bin(check_spectrum(l, 1), check_spectrum(l, 2), '/')); return 1; }
static int spec_eq(lua_State* l) {
  bool eq = luaL_testudata(l, 1, SPEC_T) && luaL_testudata(l, 2, SPEC_T);
  if(eq) {
    Spectrum a = check_spectrum(l, 1), b = check_spectrum(l, 2);
    eq = a.r == b.r && a.g == b.g && a.b == b.b;
  }
  lua_pushboolean(l, eq);
  return 1;
}
static int spec_r(lua_State* l) { lua_pushnumber(l, check_spectrum(l, 1).r); return 1; }
static int spec_g(lua_State* l) { lua_pushnumber(l, check_spectrum(l, 1).g); return 1; }
static int spec_b(lua_State* l) { lua_pushnumber(l, check_spectrum(l, 1).b); return 1; }
static int spec_tostring(lua_State* l) {
  Spectrum s = check_spectrum(l, 1);
  lua_pushfstring(l, "rgb(%f, %f, %f)", s.r, s.g, s.b);
  return 1;
}

int open_spectrum(lua_State* l) {
  const luaL_Reg methods[] = {
      {"r", spec_r}, {"g", spec_g}, {"b", spec_b}, {"red", spec_r}, {"green", spec_g},
      {"blue", spec_b}, {"__add", spec_add}, {"__sub", spec_sub}, {"__mul", spec_mul},
      {"__div", spec_div}, {"__eq", spec_eq}, {"__tostring", spec_tostring},
      {nullptr, nullptr}};
  register_type(l, SPEC_T, methods, nullptr);
  const luaL_Reg funs[] = {{"rgb", spec_rgb}, {"rgbh", spec_rgbh}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- dort.math (lua_math.cpp) -------------------------------------------------------

constexpr const char* RNG_T = "dort.Rng";

template<double (*F)(double)>
static int math_unary(lua_State* l) { lua_pushnumber(l, F(luaL_checknumber(l, 1))); return 1; }
template<double (*F)(double, double)>
static int math_binary(lua_State* l) {
  lua_pushnumber(l, F(luaL_checknumber(l, 1), luaL_checknumber(l, 2)));
  return 1;
}
static double sq(double x) { return x * x; }
static double dabs(double x) { return std::fabs(x); }
static double dsqrt(double x) { return std::sqrt(x); }
static double dexp(double x) { return std::exp(x); }
static double dfloor(double x) { return std::floor(x); }
static double dceil(double x) { return std::ceil(x); }
static double dsin(double x) { return std::sin(x); }
static double dcos(double x) { return std::cos(x); }
static double dtan(double x) { return std::tan(x); }
static double dasin(double x) { return std::asin(x); }
static double dacos(double x) { return std::acos(x); }
static double datan2(double y, double x) { return std::atan2(y, x); }
static double dpow(double x, double y) { return std::pow(x, y); }

static int math_min(lua_State* l) {
  double m = INFINITY;
  for(int i = 1; i <= lua_gettop(l); ++i) { m = std::fmin(m, luaL_checknumber(l, i)); }
  lua_pushnumber(l, m);
  return 1;
}
static int math_max(lua_State* l) {
  double m = -INFINITY;
  for(int i = 1; i <= lua_gettop(l); ++i) { m = std::fmax(m, luaL_checknumber(l, i)); }
  lua_pushnumber(l, m);
  return 1;
}

// The reference's Rng (include/dort/rng.hpp): a standard mt19937 drawing
// uniform floats with the standard library's distribution, so scripts that
// generate geometry from a seed get the same geometry.
static int math_make_rng(lua_State* l) {
  uint32_t seed = uint32_t(luaL_checkinteger(l, 1));
  push_shared(l, RNG_T, std::make_shared<std::mt19937>(seed));
  return 1;
}
static int rng_call(lua_State* l) {
  auto g = check_shared<std::mt19937>(l, 1, RNG_T);
  float lo = lua_gettop(l) >= 2 ? float(luaL_checknumber(l, 2)) : 0.f;
  float hi = lua_gettop(l) >= 3 ? float(luaL_checknumber(l, 3)) : 1.f;
  float u = std::uniform_real_distribution<float>(0.f, 1.f)(*g);
  lua_pushnumber(l, u * (hi - lo) + lo);
  return 1;
}

int open_math(lua_State* l) {
  const luaL_Reg rng_methods[] = {{"__call", rng_call}, {nullptr, nullptr}};
  register_type(l, RNG_T, rng_methods, gc_shared<std::mt19937>);
  const luaL_Reg funs[] = {
      {"sqrt", math_unary<dsqrt>}, {"exp", math_unary<dexp>}, {"floor", math_unary<dfloor>},
      {"ceil", math_unary<dceil>}, {"abs", math_unary<dabs>}, {"sin", math_unary<dsin>},
      {"cos", math_unary<dcos>}, {"tan", math_unary<dtan>}, {"asin", math_unary<dasin>},
      {"acos", math_unary<dacos>}, {"atan2", math_binary<datan2>},
      {"square", math_unary<sq>}, {"pow", math_binary<dpow>}, {"min", math_min},
      {"max", math_max}, {"make_rng", math_make_rng}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  lua_pushnumber(l, INFINITY);
  lua_setfield(l, -2, "infinity");
  lua_pushnumber(l, 3.14159265358979323846);
  lua_setfield(l, -2, "pi");
  lua_pushnumber(l, 6.28318530717958647692);
  lua_setfield(l, -2, "two_pi");
  return 1;
}

}  // namespace dortlua
