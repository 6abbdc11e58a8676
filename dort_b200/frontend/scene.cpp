// Scene description of the Lua front-end: dort.shape, dort.material,
// dort.light, dort.camera, dort.texture and dort.builder (the reference's
// lua_shape.cpp, lua_material.cpp, lua_light.cpp, lua_camera.cpp,
// lua_builder.cpp), and the flattening of a built scene into the C ABI's
// dort_scene_desc.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "frontend.h"

namespace dortlua {

// ---- shapes and meshes ---------------------------------------------------------------

static std::shared_ptr<Shape> check_shape(lua_State* l, int idx) {
  return check_shared<Shape>(l, idx, SHAPE_T);
}

static int push_shape(lua_State* l, std::shared_ptr<Shape> s) {
  push_shared(l, SHAPE_T, std::move(s));
  return 1;
}

static int shape_sphere(lua_State* l) {
  int p = params_index(l, 1);
  auto s = std::make_shared<Shape>();
  s->kind = DORT_SHAPE_SPHERE;
  s->param[0] = param_number(l, p, "radius");
  params_check_unused(l, p);
  return push_shape(l, s);
}

static int shape_disk(lua_State* l) {
  int p = params_index(l, 1);
  auto s = std::make_shared<Shape>();
  s->kind = DORT_SHAPE_DISK;
  s->param[0] = param_number(l, p, "radius");
  s->param[1] = param_number_opt(l, p, "z", 0.0);
  params_check_unused(l, p);
  return push_shape(l, s);
}

static int shape_cylinder(lua_State* l) {
  int p = params_index(l, 1);
  auto s = std::make_shared<Shape>();
  s->kind = DORT_SHAPE_CYLINDER;
  s->param[0] = param_number(l, p, "radius");
  s->param[1] = param_number_opt(l, p, "z_min", -1.0);
  s->param[2] = param_number_opt(l, p, "z_max", 1.0);
  params_check_unused(l, p);
  return push_shape(l, s);
}

static int shape_cube(lua_State* l) {
  auto s = std::make_shared<Shape>();
  s->kind = DORT_SHAPE_CUBE;
  return push_shape(l, s);
}

static int shape_polygon(lua_State* l) {
  return luaL_error(l, "polygon shapes are not supported by this renderer");
}

static double shape_area_of(const Shape& s) {
  const double pi = 3.14159265358979323846;
  switch(s.kind) {
    case DORT_SHAPE_SPHERE: return 4.0 * pi * s.param[0] * s.param[0];
    case DORT_SHAPE_DISK: return pi * s.param[0] * s.param[0];
    case DORT_SHAPE_CUBE: return 24.0;
    case DORT_SHAPE_CYLINDER: return 2.0 * pi * s.param[0] * (s.param[2] - s.param[1]);
    default: {
      const Mesh& m = *s.mesh;
      V3 a = m.points[m.vertices[s.index]], b = m.points[m.vertices[s.index + 1]];
      V3 c = m.points[m.vertices[s.index + 2]];
      V3 e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{c.x - a.x, c.y - a.y, c.z - a.z};
      V3 n{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
      return 0.5 * std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    }
  }
}

static int shape_get_area(lua_State* l) {
  lua_pushnumber(l, shape_area_of(*check_shape(l, 1)));
  return 1;
}

// lua_shape.cpp: make_mesh{points, vertices, transform}; the points are taken
// through the transform when the mesh is made
static int shape_mesh(lua_State* l) {
  int p = params_index(l, 1);
  Transform t = param_transform_opt(l, p, "transform", Transform::identity());
  auto mesh = std::make_shared<Mesh>();
  if(!param_take(l, p, "points")) { return luaL_error(l, "Missing parameter 'points'"); }
  luaL_checktype(l, -1, LUA_TTABLE);
  lua_Integer np = luaL_len(l, -1);
  for(lua_Integer i = 1; i <= np; ++i) {
    lua_rawgeti(l, -1, i);
    mesh->points.push_back(t.mat.point(check_vec3(l, -1, KIND_POINT)));
    lua_pop(l, 1);
  }
  lua_pop(l, 1);
  if(param_take(l, p, "uvs")) { lua_pop(l, 1); }   // texture coordinates: unused here
  if(param_take(l, p, "normals")) {
    return luaL_error(l, "per-vertex normals are not supported by this renderer");
  }
  if(!param_take(l, p, "vertices")) { return luaL_error(l, "Missing parameter 'vertices'"); }
  luaL_checktype(l, -1, LUA_TTABLE);
  lua_Integer nv = luaL_len(l, -1);
  for(lua_Integer i = 1; i <= nv; ++i) {
    lua_rawgeti(l, -1, i);
    lua_Integer v = luaL_checkinteger(l, -1);
    if(v < 0 || v >= lua_Integer(mesh->points.size())) {
      return luaL_error(l, "vertex index %d out of range", int(v));
    }
    mesh->vertices.push_back(uint32_t(v));
    lua_pop(l, 1);
  }
  lua_pop(l, 1);
  params_check_unused(l, p);
  push_shared(l, MESH_T, mesh);
  return 1;
}

// PLY reading as the reference's read_ply_callbacks (ply_mesh.cpp:9-78, over
// rply): ascii and binary little / big endian; x / y / z of "vertex" update
// one persistent point, emitted (rounded to float) when z is read; the
// "vertex_indices" list of "face" fanned into triangles (i0, i_{j-1}, i_j).
// An index past the points is an error here (the reference reads out of
// bounds later).
static bool read_ply(const char* path, const Transform& t, Mesh& out, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if(!f) { err = std::string("Could not open ply mesh file for reading: ") + path; return false; }
  auto fail = [&](const std::string& why) {
    err = std::string("Could not read ply file: ") + path + " (" + why + ")";
    return false;
  };
  std::string line;
  std::getline(f, line);
  if(line.rfind("ply", 0) != 0) { return fail("not a PLY file"); }
  enum Fmt { ASCII, BLE, BBE } fmt = ASCII;
  struct Prop { std::string name, type, count_type; bool list = false; };
  struct Elem { std::string name; uint64_t count = 0; std::vector<Prop> props; };
  std::vector<Elem> elems;
  while(std::getline(f, line)) {
    if(!line.empty() && line.back() == '\r') { line.pop_back(); }
    std::istringstream ss(line);
    std::string w;
    ss >> w;
    if(w == "format") {
      std::string fm;
      ss >> fm;
      if(fm == "ascii") { fmt = ASCII; }
      else if(fm == "binary_little_endian") { fmt = BLE; }
      else if(fm == "binary_big_endian") { fmt = BBE; }
      else { return fail("unknown PLY format " + fm); }
    } else if(w == "element") {
      Elem e;
      ss >> e.name >> e.count;
      elems.push_back(e);
    } else if(w == "property") {
      if(elems.empty()) { return fail("PLY property before element"); }
      Prop pr;
      ss >> pr.type;
      if(pr.type == "list") { pr.list = true; ss >> pr.count_type >> pr.type; }
      ss >> pr.name;
      elems.back().props.push_back(pr);
    } else if(w == "end_header") {
      break;
    }
  }
  auto type_size = [](const std::string& ty) -> int {
    if(ty == "char" || ty == "uchar" || ty == "int8" || ty == "uint8") { return 1; }
    if(ty == "short" || ty == "ushort" || ty == "int16" || ty == "uint16") { return 2; }
    if(ty == "int" || ty == "uint" || ty == "float" || ty == "int32" || ty == "uint32" ||
       ty == "float32") { return 4; }
    if(ty == "double" || ty == "float64") { return 8; }
    return 0;
  };
  auto read_bin = [&](const std::string& ty, double& v) -> bool {
    int n = type_size(ty);
    unsigned char b[8];
    if(n == 0 || !f.read(reinterpret_cast<char*>(b), n)) { return false; }
    if(fmt == BBE) { for(int i = 0; i < n / 2; ++i) { std::swap(b[i], b[n - 1 - i]); } }
    if(ty == "char" || ty == "int8") { v = double(int8_t(b[0])); }
    else if(ty == "uchar" || ty == "uint8") { v = double(b[0]); }
    else if(ty == "short" || ty == "int16") { int16_t x; std::memcpy(&x, b, 2); v = x; }
    else if(ty == "ushort" || ty == "uint16") { uint16_t x; std::memcpy(&x, b, 2); v = x; }
    else if(ty == "int" || ty == "int32") { int32_t x; std::memcpy(&x, b, 4); v = x; }
    else if(ty == "uint" || ty == "uint32") { uint32_t x; std::memcpy(&x, b, 4); v = x; }
    else if(ty == "float" || ty == "float32") { float x; std::memcpy(&x, b, 4); v = x; }
    else { double x; std::memcpy(&x, b, 8); v = x; }
    return true;
  };
  auto read_val = [&](const std::string& ty, double& v) -> bool {
    if(fmt == ASCII) { return bool(f >> v); }
    return read_bin(ty, v);
  };
  size_t base = out.points.size();
  float xyz[3] = {0, 0, 0};
  for(const Elem& e : elems) {
    for(uint64_t k = 0; k < e.count; ++k) {
      std::vector<uint32_t> face;
      for(const Prop& pr : e.props) {
        if(pr.list) {
          double cnt;
          if(!read_val(pr.count_type, cnt)) { return fail("truncated PLY file"); }
          for(int64_t j = 0; j < int64_t(cnt); ++j) {
            double v;
            if(!read_val(pr.type, v)) { return fail("truncated PLY file"); }
            if(e.name == "face" && pr.name == "vertex_indices") { face.push_back(uint32_t(v)); }
          }
        } else {
          double v;
          if(!read_val(pr.type, v)) { return fail("truncated PLY file"); }
          if(e.name == "vertex") {
            if(pr.name == "x") { xyz[0] = float(v); } else if(pr.name == "y") { xyz[1] = float(v); }
            else if(pr.name == "z") {
              xyz[2] = float(v);
              out.points.push_back(t.mat.point(V3{xyz[0], xyz[1], xyz[2]}));
            }
          }
        }
      }
      if(e.name == "face") {
        for(size_t j = 2; j < face.size(); ++j) {
          out.vertices.push_back(uint32_t(base + face[0]));
          out.vertices.push_back(uint32_t(base + face[j - 1]));
          out.vertices.push_back(uint32_t(base + face[j]));
        }
      }
    }
  }
  for(uint32_t v : out.vertices) {
    if(v >= out.points.size()) { return fail("PLY face index out of range"); }
  }
  return true;
}

static int shape_read_ply_mesh(lua_State* l) {
  const char* path = luaL_checkstring(l, 1);
  auto mesh = std::make_shared<Mesh>();
  std::string err;
  if(!read_ply(path, Transform::identity(), *mesh, err)) { return luaL_error(l, "%s", err.c_str()); }
  push_shared(l, MESH_T, mesh);
  return 1;
}

int open_shape(lua_State* l) {
  const luaL_Reg shape_methods[] = {{"get_area", shape_get_area}, {nullptr, nullptr}};
  register_type(l, SHAPE_T, shape_methods, gc_shared<Shape>);
  const luaL_Reg mesh_methods[] = {{nullptr, nullptr}};
  register_type(l, MESH_T, mesh_methods, gc_shared<Mesh>);
  const luaL_Reg funs[] = {
      {"get_area", shape_get_area}, {"make_sphere", shape_sphere}, {"make_disk", shape_disk},
      {"make_cylinder", shape_cylinder}, {"make_cube", shape_cube},
      {"make_polygon", shape_polygon}, {"make_mesh", shape_mesh},
      {"read_ply_mesh", shape_read_ply_mesh}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- materials (lua_material.cpp; defaults as there) ---------------------------------

static int push_material(lua_State* l, const dort_material& m) {
  auto mat = std::make_shared<Material>();
  mat->m = m;
  push_shared(l, MAT_T, mat);
  return 1;
}

static void set_rgb(float* dst, Spectrum s) { dst[0] = float(s.r); dst[1] = float(s.g); dst[2] = float(s.b); }

static int mat_lambert(lua_State* l) {
  int p = params_index(l, 1);
  dort_material m{};
  m.kind = DORT_MAT_LAMBERT;
  set_rgb(m.color, param_spectrum_opt(l, p, "albedo", {1, 1, 1}));
  params_check_unused(l, p);
  return push_material(l, m);
}

static int mat_oren_nayar(lua_State* l) {
  int p = params_index(l, 1);
  dort_material m{};
  m.kind = DORT_MAT_OREN_NAYAR;
  set_rgb(m.color, param_spectrum_opt(l, p, "albedo", {1, 1, 1}));
  m.param[0] = float(param_number_opt(l, p, "sigma", 0.1));
  params_check_unused(l, p);
  return push_material(l, m);
}

static int mat_mirror(lua_State* l) {
  int p = params_index(l, 1);
  dort_material m{};
  m.kind = DORT_MAT_MIRROR;
  set_rgb(m.color, param_spectrum_opt(l, p, "albedo", {1, 1, 1}));
  params_check_unused(l, p);
  return push_material(l, m);
}

static int mat_dielectric(lua_State* l) {
  int p = params_index(l, 1);
  dort_material m{};
  m.kind = DORT_MAT_DIELECTRIC;
  set_rgb(m.color, param_spectrum_opt(l, p, "reflect_tint", {1, 1, 1}));
  set_rgb(m.color2, param_spectrum_opt(l, p, "transmit_tint", {1, 1, 1}));
  m.param[0] = float(param_number_opt(l, p, "ior_inside", 1.5));
  m.param[1] = float(param_number_opt(l, p, "ior_outside", 1.0));
  m.param[2] = param_bool_opt(l, p, "is_thin", false) ? 1.f : 0.f;
  if(m.param[0] == 0.f || m.param[1] == 0.f) {
    // a zero ior means "no BxDF" in the reference (dielectric_material.cpp:108);
    // the C ABI reads 0 as the default, so pass a negative value instead
    if(m.param[0] == 0.f) { m.param[0] = -1.f; }
    if(m.param[1] == 0.f) { m.param[1] = -1.f; }
  }
  params_check_unused(l, p);
  return push_material(l, m);
}

static int mat_phong(lua_State* l) {
  int p = params_index(l, 1);
  dort_material m{};
  m.kind = DORT_MAT_PHONG;
  Spectrum diffuse = param_spectrum_opt(l, p, "albedo", {0, 0, 0});
  set_rgb(m.color, diffuse);
  set_rgb(m.color2, param_spectrum_opt(l, p, "glossy_albedo", diffuse));
  m.param[0] = float(param_number_opt(l, p, "exponent", 50.0));
  params_check_unused(l, p);
  return push_material(l, m);
}

static int mat_unsupported(lua_State* l) {
  return luaL_error(l, "this material is not supported by this renderer");
}

int open_material(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, MAT_T, methods, gc_shared<Material>);
  const luaL_Reg funs[] = {
      {"make_lambert", mat_lambert}, {"make_oren_nayar", mat_oren_nayar},
      {"make_mirror", mat_mirror}, {"make_dielectric", mat_dielectric},
      {"make_phong", mat_phong}, {"make_rough_dielectric", mat_unsupported},
      {"make_bump", mat_unsupported}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// Textures: only constants (numbers and spectra passed directly) are
// supported; the texture constructors report that.
static int tex_unsupported(lua_State* l) {
  return luaL_error(l, "textures other than constants are not supported by this renderer");
}

int open_texture(lua_State* l) {
  static const char* names[] = {
      "compose", "make_const_geom", "make_const_1d", "make_const_2d", "make_const_3d",
      "make_identity_1d", "make_identity_2d", "make_identity_3d", "make_lerp",
      "make_checkerboard_1d", "make_checkerboard_2d", "make_checkerboard_3d",
      "make_value_noise_1d", "make_value_noise_2d", "make_value_noise_3d",
      "make_value_noise_1d_of_2d", "make_value_noise_2d_of_2d", "make_value_noise_3d_of_2d",
      "make_value_noise_1d_of_3d", "make_value_noise_2d_of_3d", "make_value_noise_3d_of_3d",
      "make_image", "make_gain", "make_bias", "make_map_uv", "make_map_xy",
      "make_map_spherical", "make_map_cylindrical", "make_map_xyz",
      "make_color_map_grayscale", "make_color_map_lerp", "make_color_map_spline",
      "render_2d", nullptr};
  lua_newtable(l);
  for(int i = 0; names[i]; ++i) {
    lua_pushcfunction(l, tex_unsupported);
    lua_setfield(l, -2, names[i]);
  }
  return 1;
}

// ---- lights (lua_light.cpp) --------------------------------------------------------------

static int push_light(lua_State* l, std::shared_ptr<Light> li) {
  push_shared(l, LIGHT_T, std::move(li));
  return 1;
}

static int light_point(lua_State* l) {
  int p = params_index(l, 1);
  auto li = std::make_shared<Light>();
  li->kind = Light::POINT;
  V3 pt = param_vec3(l, p, "point", KIND_POINT);
  li->rgb = param_spectrum(l, p, "intensity");
  Transform t = param_transform_opt(l, p, "transform", Transform::identity());
  li->vec = t.mat.point(pt);
  params_check_unused(l, p);
  return push_light(l, li);
}

static int light_directional(lua_State* l) {
  int p = params_index(l, 1);
  auto li = std::make_shared<Light>();
  li->kind = Light::DIRECTIONAL;
  V3 d = param_vec3(l, p, "direction", KIND_VECTOR);
  li->rgb = param_spectrum(l, p, "radiance");
  Transform t = param_transform_opt(l, p, "transform", Transform::identity());
  li->vec = t.mat.vector(d);
  params_check_unused(l, p);
  return push_light(l, li);
}

static int light_diffuse(lua_State* l) {
  int p = params_index(l, 1);
  auto li = std::make_shared<Light>();
  li->kind = Light::DIFFUSE;
  if(!param_take(l, p, "shape")) { return luaL_error(l, "Missing parameter 'shape'"); }
  li->shape = check_shape(l, -1);
  lua_pop(l, 1);
  li->rgb = param_spectrum(l, p, "radiance");
  li->transform = param_transform_opt(l, p, "transform", Transform::identity());
  params_check_unused(l, p);
  return push_light(l, li);
}

static int light_infinite(lua_State* l) {
  int p = params_index(l, 1);
  auto li = std::make_shared<Light>();
  li->kind = Light::INFINITE;
  li->rgb = param_spectrum(l, p, "radiance");
  params_check_unused(l, p);
  return push_light(l, li);
}

static int light_environment(lua_State* l) {
  int p = params_index(l, 1);
  auto li = std::make_shared<Light>();
  li->kind = Light::ENVIRONMENT;
  if(!param_take(l, p, "image")) { return luaL_error(l, "Missing parameter 'image'"); }
  li->image = check_image(l, -1);
  lua_pop(l, 1);
  if(!li->image->hdr) { return luaL_error(l, "the environment image must be an HDR image"); }
  V3 up = param_vec3(l, p, "up", KIND_VECTOR);
  V3 fwd = param_vec3(l, p, "forward", KIND_VECTOR);
  li->rgb = param_spectrum_opt(l, p, "scale", {1, 1, 1});
  Transform t = param_transform_opt(l, p, "transform", Transform::identity());
  li->up = t.mat.vector(up);
  li->forward = t.mat.vector(fwd);
  params_check_unused(l, p);
  return push_light(l, li);
}

static int light_beam(lua_State* l) {
  return luaL_error(l, "beam lights are invisible to the \"pt\" renderer and not supported");
}

int open_light(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, LIGHT_T, methods, gc_shared<Light>);
  const luaL_Reg funs[] = {
      {"make_point", light_point}, {"make_directional", light_directional},
      {"make_diffuse", light_diffuse}, {"make_infinite", light_infinite},
      {"make_environment", light_environment}, {"make_beam", light_beam},
      {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- cameras (lua_camera.cpp) ----------------------------------------------------------------

static void camera_columns(dort_camera& c, const Transform& t) {
  for(int r = 0; r < 3; ++r) {
    c.right[r] = float(t.mat.m[r][0]);
    c.up[r] = float(t.mat.m[r][1]);
    c.forward[r] = float(t.mat.m[r][2]);
    c.origin[r] = float(t.mat.m[r][3]);
  }
}

static int push_camera(lua_State* l, const dort_camera& c) {
  auto cam = std::make_shared<Camera>();
  cam->c = c;
  push_shared(l, CAM_T, cam);
  return 1;
}

static int camera_pinhole(lua_State* l) {
  int p = params_index(l, 1);
  dort_camera c{};
  c.kind = DORT_CAMERA_PINHOLE;
  camera_columns(c, param_transform(l, p, "transform"));
  c.fov = float(param_number_opt(l, p, "fov", 3.14159265358979323846 * 0.5));
  params_check_unused(l, p);
  return push_camera(l, c);
}

static int camera_ortho(lua_State* l) {
  int p = params_index(l, 1);
  dort_camera c{};
  c.kind = DORT_CAMERA_ORTHO;
  camera_columns(c, param_transform_opt(l, p, "transform", Transform::identity()));
  c.dimension = float(param_number(l, p, "dimension"));
  params_check_unused(l, p);
  return push_camera(l, c);
}

static int camera_thin_lens(lua_State* l) {
  int p = params_index(l, 1);
  dort_camera c{};
  c.kind = DORT_CAMERA_THIN_LENS;
  camera_columns(c, param_transform(l, p, "transform"));
  c.lens_radius = float(param_number(l, p, "lens_radius"));
  c.focal_distance = float(param_number(l, p, "focal_distance"));
  c.fov = float(param_number_opt(l, p, "fov", 3.14159265358979323846 * 0.5));
  params_check_unused(l, p);
  return push_camera(l, c);
}

int open_camera(lua_State* l) {
  const luaL_Reg methods[] = {{nullptr, nullptr}};
  register_type(l, CAM_T, methods, gc_shared<Camera>);
  const luaL_Reg funs[] = {
      {"make_pinhole", camera_pinhole}, {"make_ortho", camera_ortho},
      {"make_thin_lens", camera_thin_lens}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- the builder (lua_builder.cpp) ----------------------------------------------------------

static std::shared_ptr<Builder> check_builder(lua_State* l, int idx) {
  return check_shared<Builder>(l, idx, BUILDER_T);
}

static int b_make(lua_State* l) {
  push_shared(l, BUILDER_T, std::make_shared<Builder>());
  return 1;
}

static int b_push_state(lua_State* l) {
  auto b = check_builder(l, 1);
  b->state_stack.push_back(b->state);
  return 0;
}

static int b_pop_state(lua_State* l) {
  auto b = check_builder(l, 1);
  if(b->state_stack.empty()) { return luaL_error(l, "State stack is empty (not balanced)"); }
  b->state = b->state_stack.back();
  b->state_stack.pop_back();
  return 0;
}

// lua_builder.cpp:177-220: a frame starts with an identity transform and the
// current material
static int b_push_frame(lua_State* l) {
  auto b = check_builder(l, 1);
  BuilderState fresh;
  fresh.material = b->state.material;
  b->state_stack.push_back(b->state);
  b->frame_stack.push_back(std::move(b->frame));
  b->state = fresh;
  b->frame.clear();
  return 0;
}

static int b_pop_frame(lua_State* l) {
  auto b = check_builder(l, 1);
  if(b->frame_stack.empty()) { return luaL_error(l, "Frame stack is empty (not balanced)"); }
  if(b->state_stack.empty()) { return luaL_error(l, "State stack is empty (not balanced)"); }
  auto fr = std::make_shared<FramePrim>();
  fr->prims = std::make_shared<PrimList>(std::move(b->frame));
  b->frame = std::move(b->frame_stack.back());
  b->frame_stack.pop_back();
  b->state = b->state_stack.back();
  b->state_stack.pop_back();
  push_shared(l, FRAME_T, fr);
  return 1;
}

// lua_builder.cpp:227-232: composes with the current transform
static int b_set_transform(lua_State* l) {
  auto b = check_builder(l, 1);
  b->state.local_to_frame = b->state.local_to_frame * check_transform(l, 2);
  return 0;
}

static int b_get_transform(lua_State* l) {
  push_transform(l, check_builder(l, 1)->state.local_to_frame);
  return 1;
}

static int b_set_material(lua_State* l) {
  check_builder(l, 1)->state.material = check_shared<Material>(l, 2, MAT_T);
  return 0;
}

static int b_get_material(lua_State* l) {
  auto b = check_builder(l, 1);
  if(!b->state.material) { lua_pushnil(l); return 1; }
  push_shared(l, MAT_T, b->state.material);
  return 1;
}

static int b_set_camera(lua_State* l) {
  check_builder(l, 1)->camera = check_shared<Camera>(l, 2, CAM_T);
  return 0;
}

static int b_get_scene_default_camera(lua_State* l);

static int b_set_option(lua_State* l) {
  auto b = check_builder(l, 1);
  std::string opt = luaL_checkstring(l, 2);
  if(opt == "bvh_split_method") {
    std::string m = luaL_checkstring(l, 3);
    if(m != "sah" && m != "middle") { return luaL_error(l, "unknown bvh split method: %s", m.c_str()); }
    // the device BVH is always built with binned SAH
  } else if(opt == "bvh_leaf_size" || opt == "bvh_max_leaf_size") {
    luaL_checkinteger(l, 3);   // leaf sizes of the wide BVH are fixed
  } else {
    return luaL_error(l, "unknown option: %s", opt.c_str());
  }
  (void)b;
  return 0;
}

static void need_material(lua_State* l, const Builder& b) {
  if(!b.state.material) { luaL_error(l, "no material is set"); }
}

static int b_add_shape(lua_State* l) {
  auto b = check_builder(l, 1);
  Prim pr;
  pr.kind = Prim::SHAPE;
  pr.shape = check_shape(l, 2);
  need_material(l, *b);
  pr.material = b->state.material;
  pr.transform = b->state.local_to_frame;
  if(lua_gettop(l) >= 3 && !lua_isnil(l, 3)) {
    pr.light = check_shared<Light>(l, 3, LIGHT_T);
    if(pr.light->kind != Light::DIFFUSE) { return luaL_error(l, "the light must be an area light"); }
  }
  b->frame.push_back(pr);
  return 0;
}

static int b_add_primitive(lua_State* l) {
  auto b = check_builder(l, 1);
  auto fr = check_shared<FramePrim>(l, 2, FRAME_T);
  Prim pr;
  pr.kind = Prim::INSTANCE;
  pr.frame = fr->prims;
  pr.transform = b->state.local_to_frame;
  b->frame.push_back(pr);
  return 0;
}

static std::shared_ptr<Shape> triangle_shape(lua_State* l, std::shared_ptr<Mesh> mesh,
                                             lua_Integer index) {
  if(index < 0 || size_t(index) + 3 > mesh->vertices.size()) {
    luaL_error(l, "triangle index %d out of range", int(index));
  }
  auto s = std::make_shared<Shape>();
  s->kind = SHAPE_TRIANGLE;
  s->mesh = std::move(mesh);
  s->index = uint32_t(index);
  return s;
}

// lua_builder.cpp:368-391: the mesh's coordinates are used directly
static int b_add_triangle(lua_State* l) {
  auto b = check_builder(l, 1);
  auto mesh = check_shared<Mesh>(l, 2, MESH_T);
  need_material(l, *b);
  Prim pr;
  pr.kind = Prim::TRIANGLE;
  pr.shape = triangle_shape(l, mesh, luaL_checkinteger(l, 3));
  pr.material = b->state.material;
  b->frame.push_back(pr);
  return 0;
}

static int b_make_triangle(lua_State* l) {
  check_builder(l, 1);
  auto mesh = check_shared<Mesh>(l, 2, MESH_T);
  push_shared(l, SHAPE_T, triangle_shape(l, mesh, luaL_checkinteger(l, 3)));
  return 1;
}

static int b_add_light(lua_State* l) {
  auto b = check_builder(l, 1);
  if(!b->frame_stack.empty()) { return luaL_error(l, "lights can only be added in the root frame"); }
  b->lights.push_back(check_shared<Light>(l, 2, LIGHT_T));
  return 0;
}

// every triangle of a mesh as its own primitive with the current material
static void add_mesh_triangles(lua_State* l, Builder& b, std::shared_ptr<Mesh> mesh) {
  need_material(l, b);
  for(size_t i = 0; i + 2 < mesh->vertices.size(); i += 3) {
    Prim pr;
    pr.kind = Prim::TRIANGLE;
    pr.shape = triangle_shape(l, mesh, lua_Integer(i));
    pr.material = b.state.material;
    b.frame.push_back(pr);
  }
}

// lua_builder.cpp:418-564: PLY meshes with the current transform applied to
// their points; "as_bvh" (one BVH per mesh in the reference) is the same set
// of triangles here
static int b_add_read_ply_mesh(lua_State* l) {
  auto b = check_builder(l, 1);
  const char* path = luaL_checkstring(l, 2);
  auto mesh = std::make_shared<Mesh>();
  std::string err;
  if(!read_ply(path, b->state.local_to_frame, *mesh, err)) { return luaL_error(l, "%s", err.c_str()); }
  add_mesh_triangles(l, *b, mesh);
  return 0;
}

static int b_add_ply_mesh(lua_State* l) {
  auto b = check_builder(l, 1);
  auto src = check_shared<Mesh>(l, 2, MESH_T);
  auto mesh = std::make_shared<Mesh>();
  for(const V3& p : src->points) { mesh->points.push_back(b->state.local_to_frame.mat.point(p)); }
  mesh->vertices = src->vertices;
  add_mesh_triangles(l, *b, mesh);
  return 0;
}

static int b_add_voxel_grid(lua_State* l) {
  return luaL_error(l, "voxel grids are not supported by this renderer");
}

// ---- flattening (build_scene, lua_builder.cpp:113-146) ----------------------------------

namespace {

struct Flattener {
  lua_State* l;
  FlatScene& f;
  std::map<const Material*, uint32_t> mat_ids;
  std::map<const Light*, bool> lit;

  uint32_t mat_id(const std::shared_ptr<Material>& m) {
    auto it = mat_ids.find(m.get());
    if(it != mat_ids.end()) { return it->second; }
    uint32_t id = uint32_t(f.materials.size());
    f.materials.push_back(m->m);
    mat_ids[m.get()] = id;
    return id;
  }

  void emit(const PrimList& prims, const Transform& outer) {
    for(const Prim& p : prims) {
      if(p.kind == Prim::INSTANCE) {
        emit(*p.frame, outer * p.transform);
        continue;
      }
      Spectrum em{0, 0, 0};
      bool light_differs = false;
      if(p.light) {
        em = p.light->rgb;
        lit[p.light.get()] = true;
        light_differs = !(p.light->transform.mat == (outer * p.transform).mat);
      }
      if(p.shape->kind == SHAPE_TRIANGLE) {
        Transform t = p.kind == Prim::TRIANGLE ? outer : outer * p.transform;
        const Mesh& m = *p.shape->mesh;
        uint32_t base = uint32_t(f.verts.size() / 3);
        for(int k = 0; k < 3; ++k) {
          V3 src = m.points[m.vertices[p.shape->index + k]];
          V3 q = t.mat.point(src);
          f.verts.push_back(float(q.x));
          f.verts.push_back(float(q.y));
          f.verts.push_back(float(q.z));
          f.tris.push_back(base + uint32_t(k));
          // the triangle the light samples: the shape under the light's own
          // transform (the same points unless the transforms differ)
          V3 lq = (p.light && light_differs) ? p.light->transform.mat.point(src) : q;
          f.tri_light_verts.push_back(float(lq.x));
          f.tri_light_verts.push_back(float(lq.y));
          f.tri_light_verts.push_back(float(lq.z));
        }
        if(p.light && light_differs) { f.light_verts_used = true; }
        f.tri_material.push_back(mat_id(p.material));
        f.tri_emission.push_back(float(em.r));
        f.tri_emission.push_back(float(em.g));
        f.tri_emission.push_back(float(em.b));
      } else {
        Transform t = outer * p.transform;
        dort_shape s{};
        s.kind = p.shape->kind;
        s.material = mat_id(p.material);
        for(int k = 0; k < 4; ++k) { s.param[k] = float(p.shape->param[k]); }
        for(int r = 0; r < 3; ++r) {
          for(int c = 0; c < 4; ++c) { s.to_world[4 * r + c] = float(t.mat.m[r][c]); }
        }
        s.emission[0] = float(em.r); s.emission[1] = float(em.g); s.emission[2] = float(em.b);
        if(p.light && light_differs) {
          s.flags |= DORT_SHAPE_LIGHT_TRANSFORM;
          for(int r = 0; r < 3; ++r) {
            for(int c = 0; c < 4; ++c) {
              s.light_to_world[4 * r + c] = float(p.light->transform.mat.m[r][c]);
            }
          }
        }
        f.shapes.push_back(s);
      }
    }
  }
};

}  // namespace

dort_scene_desc FlatScene::desc() const {
  dort_scene_desc d{};
  d.struct_size = sizeof(d);
  d.verts = verts.empty() ? nullptr : verts.data();
  d.vert_count = uint32_t(verts.size() / 3);
  d.tris = tris.empty() ? nullptr : tris.data();
  d.tri_count = uint32_t(tris.size() / 3);
  d.tri_material = tri_material.empty() ? nullptr : tri_material.data();
  d.materials = materials.empty() ? nullptr : materials.data();
  d.material_count = uint32_t(materials.size());
  d.tri_emission = tri_emission.empty() ? nullptr : tri_emission.data();
  d.tri_light_verts = light_verts_used ? tri_light_verts.data() : nullptr;
  if(sky) {
    d.sky_rgb = sky->px.data();
    d.sky_width = sky->w;
    d.sky_height = sky->h;
  }
  for(int a = 0; a < 3; ++a) {
    d.sky_const[a] = sky_const[a];
    d.sky_scale[a] = sky_scale[a];
    d.sky_up[a] = sky_up[a];
    d.sky_fwd[a] = sky_fwd[a];
  }
  d.bvh_width = bvh_width;
  d.shape_count = uint32_t(shapes.size());
  d.shapes = shapes.empty() ? nullptr : shapes.data();
  d.lights = lights.empty() ? nullptr : lights.data();
  d.light_count = uint32_t(lights.size());
  return d;
}

static int b_build_scene(lua_State* l) {
  auto b = check_builder(l, 1);
  if(!b->frame_stack.empty()) { return luaL_error(l, "Frame stack is not empty"); }
  if(!b->state_stack.empty()) { return luaL_error(l, "State stack is not empty"); }
  auto scene = std::make_shared<Scene>();
  FlatScene& f = scene->flat;
  f.bvh_width = b->bvh_width;
  Flattener fl{l, f, {}, {}};
  fl.emit(b->frame, Transform::identity());
  if(f.materials.empty()) {
    dort_material m{};
    m.kind = DORT_MAT_LAMBERT;
    m.color[0] = m.color[1] = m.color[2] = 0.5f;
    f.materials.push_back(m);
  }
  for(const auto& li : b->lights) {
    switch(li->kind) {
      case Light::POINT:
      case Light::DIRECTIONAL: {
        dort_light d{};
        d.kind = li->kind == Light::POINT ? DORT_LIGHT_POINT : DORT_LIGHT_DIRECTIONAL;
        d.rgb[0] = float(li->rgb.r); d.rgb[1] = float(li->rgb.g); d.rgb[2] = float(li->rgb.b);
        d.vec[0] = float(li->vec.x); d.vec[1] = float(li->vec.y); d.vec[2] = float(li->vec.z);
        f.lights.push_back(d);
        break;
      }
      case Light::INFINITE:
        f.sky_const[0] += float(li->rgb.r);
        f.sky_const[1] += float(li->rgb.g);
        f.sky_const[2] += float(li->rgb.b);
        break;
      case Light::ENVIRONMENT:
        if(f.sky) { return luaL_error(l, "at most one environment light is supported"); }
        f.sky = li->image;
        f.sky_scale[0] = float(li->rgb.r); f.sky_scale[1] = float(li->rgb.g);
        f.sky_scale[2] = float(li->rgb.b);
        f.sky_up[0] = float(li->up.x); f.sky_up[1] = float(li->up.y); f.sky_up[2] = float(li->up.z);
        f.sky_fwd[0] = float(li->forward.x); f.sky_fwd[1] = float(li->forward.y);
        f.sky_fwd[2] = float(li->forward.z);
        break;
      case Light::DIFFUSE:
        if(!fl.lit.count(li.get())) {
          return luaL_error(l, "a diffuse light must be added with its shape (add_shape(shape, "
                               "light)); lights without geometry are not supported");
        }
        break;
    }
  }
  scene->camera = b->camera;
  if(const char* rec = record_path()) {
    // "%d" in the path numbers the scenes of a script in build order
    static int recorded = 0;
    std::string path = rec;
    size_t at = path.find("%d");
    if(at != std::string::npos) { path.replace(at, 2, std::to_string(recorded)); }
    ++recorded;
    write_scene_json(f, b->camera.get(), path.c_str());
  } else {
    dort_scene_desc d = f.desc();
    dort_scene* h = nullptr;
    if(dort_gpu_scene_create(&d, &h) != DORT_OK) {
      return luaL_error(l, "%s", dort_gpu_last_error());
    }
    scene->handle = h;
  }
  *b = Builder();   // the builder cannot be reused (lua_builder.cpp:110-146)
  push_shared(l, SCENE_T, scene);
  return 1;
}

static int b_get_scene_default_camera(lua_State* l) {
  auto s = check_shared<Scene>(l, 1, SCENE_T);
  if(!s->camera) { lua_pushnil(l); return 1; }
  push_shared(l, CAM_T, s->camera);
  return 1;
}

int open_builder(lua_State* l) {
  const luaL_Reg empty[] = {{nullptr, nullptr}};
  register_type(l, BUILDER_T, empty, gc_shared<Builder>);
  register_type(l, FRAME_T, empty, gc_shared<FramePrim>);
  register_type(l, SCENE_T, empty, gc_shared<Scene>);
  const luaL_Reg funs[] = {
      {"make", b_make}, {"build_scene", b_build_scene}, {"push_state", b_push_state},
      {"pop_state", b_pop_state}, {"push_frame", b_push_frame}, {"pop_frame", b_pop_frame},
      {"set_transform", b_set_transform}, {"get_transform", b_get_transform},
      {"set_material", b_set_material}, {"get_material", b_get_material},
      {"set_camera", b_set_camera}, {"set_option", b_set_option},
      {"add_shape", b_add_shape}, {"add_primitive", b_add_primitive},
      {"add_triangle", b_add_triangle}, {"add_light", b_add_light},
      {"add_read_ply_mesh", b_add_read_ply_mesh}, {"add_read_ply_mesh_as_bvh", b_add_read_ply_mesh},
      {"add_ply_mesh", b_add_ply_mesh}, {"add_ply_mesh_as_bvh", b_add_ply_mesh},
      {"add_voxel_grid", b_add_voxel_grid}, {"make_triangle", b_make_triangle},
      {"get_scene_default_camera", b_get_scene_default_camera}, {nullptr, nullptr}};
  luaL_newlib(l, funs);
  return 1;
}

// ---- record mode ------------------------------------------------------------------------

const char* record_path() {
  const char* p = std::getenv("DORT_LUA_RECORD");
  return (p && *p) ? p : nullptr;
}

static void json_floats(std::FILE* o, const float* v, size_t n) {
  std::fputc('[', o);
  for(size_t i = 0; i < n; ++i) { std::fprintf(o, "%s%.9g", i ? "," : "", double(v[i])); }
  std::fputc(']', o);
}

void write_scene_json(const FlatScene& f, const Camera* cam, const char* path) {
  std::FILE* o = std::fopen(path, "w");
  if(!o) { return; }
  std::fprintf(o, "{\"verts\":");
  json_floats(o, f.verts.data(), f.verts.size());
  std::fprintf(o, ",\"tris\":[");
  for(size_t i = 0; i < f.tris.size(); ++i) { std::fprintf(o, "%s%u", i ? "," : "", f.tris[i]); }
  std::fprintf(o, "],\"tri_material\":[");
  for(size_t i = 0; i < f.tri_material.size(); ++i) {
    std::fprintf(o, "%s%u", i ? "," : "", f.tri_material[i]);
  }
  std::fprintf(o, "],\"tri_emission\":");
  json_floats(o, f.tri_emission.data(), f.tri_emission.size());
  if(f.light_verts_used) {
    std::fprintf(o, ",\"tri_light_verts\":");
    json_floats(o, f.tri_light_verts.data(), f.tri_light_verts.size());
  }
  std::fprintf(o, ",\"materials\":[");
  for(size_t i = 0; i < f.materials.size(); ++i) {
    const dort_material& m = f.materials[i];
    std::fprintf(o, "%s{\"kind\":%u,\"color\":", i ? "," : "", m.kind);
    json_floats(o, m.color, 3);
    std::fprintf(o, ",\"color2\":");
    json_floats(o, m.color2, 3);
    std::fprintf(o, ",\"param\":");
    json_floats(o, m.param, 4);
    std::fputc('}', o);
  }
  std::fprintf(o, "],\"shapes\":[");
  for(size_t i = 0; i < f.shapes.size(); ++i) {
    const dort_shape& s = f.shapes[i];
    std::fprintf(o, "%s{\"kind\":%u,\"material\":%u,\"param\":", i ? "," : "", s.kind, s.material);
    json_floats(o, s.param, 4);
    std::fprintf(o, ",\"to_world\":");
    json_floats(o, s.to_world, 12);
    std::fprintf(o, ",\"emission\":");
    json_floats(o, s.emission, 3);
    if(s.flags & DORT_SHAPE_LIGHT_TRANSFORM) {
      std::fprintf(o, ",\"light_to_world\":");
      json_floats(o, s.light_to_world, 12);
    }
    std::fputc('}', o);
  }
  std::fprintf(o, "],\"delta_lights\":[");
  for(size_t i = 0; i < f.lights.size(); ++i) {
    std::fprintf(o, "%s{\"kind\":%u,\"rgb\":", i ? "," : "", f.lights[i].kind);
    json_floats(o, f.lights[i].rgb, 3);
    std::fprintf(o, ",\"vec\":");
    json_floats(o, f.lights[i].vec, 3);
    std::fputc('}', o);
  }
  std::fprintf(o, "],\"sky_const\":");
  json_floats(o, f.sky_const, 3);
  if(cam) {
    const dort_camera& c = cam->c;
    std::fprintf(o, ",\"camera\":{\"kind\":%u,\"fov\":%.9g,\"lens_radius\":%.9g,"
                    "\"focal_distance\":%.9g,\"dimension\":%.9g,\"origin\":",
                 c.kind, double(c.fov), double(c.lens_radius), double(c.focal_distance),
                 double(c.dimension));
    json_floats(o, c.origin, 3);
    std::fprintf(o, ",\"right\":");
    json_floats(o, c.right, 3);
    std::fprintf(o, ",\"up\":");
    json_floats(o, c.up, 3);
    std::fprintf(o, ",\"forward\":");
    json_floats(o, c.forward, 3);
    std::fputc('}', o);
  }
  std::fprintf(o, "}\n");
  std::fclose(o);
}

}  // namespace dortlua
