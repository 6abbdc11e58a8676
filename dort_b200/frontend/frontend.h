// Lua front-end of the B200 path tracer: the reference renderer's scripting
// interface (the `dort` global with its builder, geometry, shape, material,
// light, camera, render and image modules; src/dort/lua_*.cpp and
// lua/dort/*.lua of the reference) implemented over the C ABI of
// include/dort_gpu.h.  Scene scripts written for the reference run unchanged
// as long as they use what this path renders ("pt" renderer, box filter,
// constant textures, triangle / sphere / disk / cube / cylinder shapes,
// area / point / directional / infinite / environment lights, pinhole /
// orthographic / thin-lens cameras).
//
// The builder records the scene the way the reference's primitive tree holds
// it and flattens it into one dort_scene_desc when the script calls
// build_scene (transforms baked into triangles, analytic shapes kept with
// their transforms), exactly as dort_b200/builder.py does in Python.
#pragma once
extern "C" {
#include "lauxlib.h"
#include "lua.h"
#include "lualib.h"
}

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "dort_gpu.h"

namespace dortlua {

// ---- values -------------------------------------------------------------------

struct V3 { double x = 0, y = 0, z = 0; };

// 4x4 affine transform with its inverse (row-major, column vectors).
struct Mat4 {
  double m[4][4];
  static Mat4 identity();
  Mat4 operator*(const Mat4& o) const;
  V3 point(V3 p) const;
  V3 vector(V3 v) const;
  Mat4 inverse() const;
  bool operator==(const Mat4& o) const;
};

struct Transform {
  Mat4 mat, inv;
  static Transform identity() { return {Mat4::identity(), Mat4::identity()}; }
  Transform operator*(const Transform& o) const { return {mat * o.mat, o.inv * inv}; }
};

struct Spectrum { double r = 0, g = 0, b = 0; };

enum VecKind { KIND_VECTOR = 0, KIND_POINT = 1, KIND_NORMAL = 2 };

// ---- scene objects --------------------------------------------------------------

struct Mesh {
  std::vector<V3> points;
  std::vector<uint32_t> vertices;
};

constexpr uint32_t SHAPE_TRIANGLE = 100;   // a triangle of a mesh (not a dort_shape kind)

struct Shape {
  uint32_t kind = 0;          // DORT_SHAPE_* or SHAPE_TRIANGLE
  double param[4] = {0, 0, 0, 0};
  std::shared_ptr<Mesh> mesh; // SHAPE_TRIANGLE
  uint32_t index = 0;         // SHAPE_TRIANGLE: first vertex index in the mesh
};

struct Material { dort_material m{}; };

struct Image {
  uint32_t w = 0, h = 0;
  bool hdr = true;            // float RGB, or 8-bit RGB stored as 0..255
  std::vector<float> px;      // w * h * 3, row 0 at the top
};

struct Light {
  enum Kind { POINT, DIRECTIONAL, DIFFUSE, INFINITE, ENVIRONMENT } kind = POINT;
  Spectrum rgb;               // intensity / radiance / scale (environment)
  V3 vec;                     // point position / direction
  std::shared_ptr<Shape> shape;   // DIFFUSE
  Transform transform = Transform::identity();   // DIFFUSE
  std::shared_ptr<Image> image;   // ENVIRONMENT
  V3 up, forward;                 // ENVIRONMENT
};

struct Camera { dort_camera c{}; };

struct Prim;
using PrimList = std::vector<Prim>;

struct Prim {
  enum Kind { TRIANGLE, SHAPE, INSTANCE } kind = TRIANGLE;
  std::shared_ptr<Shape> shape;
  std::shared_ptr<Material> material;
  std::shared_ptr<Light> light;       // area light of a SHAPE
  Transform transform = Transform::identity();
  std::shared_ptr<PrimList> frame;    // INSTANCE: the frame's primitives
};

// A frame collected by push_frame / pop_frame (dort.builder.frame).
struct FramePrim { std::shared_ptr<PrimList> prims; };

struct BuilderState {
  Transform local_to_frame = Transform::identity();
  std::shared_ptr<Material> material;
};

struct Builder {
  BuilderState state;
  std::vector<BuilderState> state_stack;
  PrimList frame;
  std::vector<PrimList> frame_stack;
  std::vector<std::shared_ptr<Light>> lights;
  std::shared_ptr<Camera> camera;
  uint32_t bvh_width = 8;
};

// The flattened scene (the arrays of a dort_scene_desc) and its device handle.
struct FlatScene {
  std::vector<float> verts;
  std::vector<uint32_t> tris, tri_material;
  std::vector<float> tri_emission;
  std::vector<float> tri_light_verts;   // 9 per triangle; used when some light differs
  bool light_verts_used = false;
  std::vector<dort_material> materials;
  std::vector<dort_shape> shapes;
  std::vector<dort_light> lights;
  float sky_const[3] = {0, 0, 0};
  std::shared_ptr<Image> sky;
  float sky_scale[3] = {0, 0, 0}, sky_up[3] = {0, 0, 0}, sky_fwd[3] = {0, 0, 0};
  uint32_t bvh_width = 8;
  dort_scene_desc desc() const;
};

struct Scene {
  FlatScene flat;
  dort_scene* handle = nullptr;       // null in record mode (no GPU)
  std::shared_ptr<Camera> camera;
  ~Scene() { if(handle) { dort_gpu_scene_destroy(handle); } }
};

struct RenderJob {
  std::shared_ptr<Scene> scene;
  dort_render_params params{};
  bool started = false, finished = false;
  bool autotune = false;              // tune the wavefront before rendering (not a
                                      // reference parameter)
  std::shared_ptr<Image> image;       // float RGB result
};

// ---- userdata -------------------------------------------------------------------

// Values are stored by value in userdata; scene objects as shared_ptr.
template<class T>
T* push_value(lua_State* l, const char* tname, const T& v) {
  void* p = lua_newuserdata(l, sizeof(T));
  T* t = new(p) T(v);
  luaL_setmetatable(l, tname);
  return t;
}

template<class T>
void push_shared(lua_State* l, const char* tname, std::shared_ptr<T> v) {
  void* p = lua_newuserdata(l, sizeof(std::shared_ptr<T>));
  new(p) std::shared_ptr<T>(std::move(v));
  luaL_setmetatable(l, tname);
}

template<class T>
std::shared_ptr<T> check_shared(lua_State* l, int idx, const char* tname) {
  return *static_cast<std::shared_ptr<T>*>(luaL_checkudata(l, idx, tname));
}

template<class T>
std::shared_ptr<T> test_shared(lua_State* l, int idx, const char* tname) {
  void* p = luaL_testudata(l, idx, tname);
  return p ? *static_cast<std::shared_ptr<T>*>(p) : nullptr;
}

template<class T>
int gc_shared(lua_State* l) {
  static_cast<std::shared_ptr<T>*>(lua_touserdata(l, 1))->~shared_ptr<T>();
  return 0;
}

// Creates the metatable `tname` with the given methods as __index (and the
// metamethods among them as metamethods).
void register_type(lua_State* l, const char* tname, const luaL_Reg* methods, lua_CFunction gc);

// Type names.
constexpr const char* VEC_T = "dort.Vector";
constexpr const char* PNT_T = "dort.Point";
constexpr const char* NRM_T = "dort.Normal";
constexpr const char* XF_T = "dort.Transform";
constexpr const char* SPEC_T = "dort.Spectrum";
constexpr const char* VEC2_T = "dort.Vec2";
constexpr const char* VEC2I_T = "dort.Vec2i";
constexpr const char* VEC3I_T = "dort.Vec3i";
constexpr const char* BOXI_T = "dort.Boxi";
constexpr const char* RECTI_T = "dort.Recti";
constexpr const char* SHAPE_T = "dort.Shape";
constexpr const char* MESH_T = "dort.Mesh";
constexpr const char* MAT_T = "dort.Material";
constexpr const char* LIGHT_T = "dort.Light";
constexpr const char* CAM_T = "dort.Camera";
constexpr const char* BUILDER_T = "dort.Builder";
constexpr const char* FRAME_T = "dort.Primitive";
constexpr const char* SCENE_T = "dort.Scene";
constexpr const char* JOB_T = "dort.RenderJob";
constexpr const char* IMAGE_T = "dort.Image";
constexpr const char* FILTER_T = "dort.Filter";
constexpr const char* SAMPLER_T = "dort.Sampler";

V3 check_vec3(lua_State* l, int idx, VecKind kind);    // exact kind
bool test_vec3(lua_State* l, int idx, VecKind kind);
void push_vec3(lua_State* l, VecKind kind, V3 v);
Transform check_transform(lua_State* l, int idx);
void push_transform(lua_State* l, const Transform& t);
Spectrum check_spectrum(lua_State* l, int idx);         // a Spectrum or a number
void push_spectrum(lua_State* l, Spectrum s);

// ---- parameter tables (lua_params.cpp semantics) ---------------------------------
// Each getter removes the key it reads, so that params_check_unused can
// report the first key nothing read: "Unused parameter '<key>'".

bool param_take(lua_State* l, int p, const char* name);   // pushes the value if present
double param_number(lua_State* l, int p, const char* name);
double param_number_opt(lua_State* l, int p, const char* name, double def);
uint32_t param_uint_opt(lua_State* l, int p, const char* name, uint32_t def);
bool param_bool_opt(lua_State* l, int p, const char* name, bool def);
std::string param_string_opt(lua_State* l, int p, const char* name, const std::string& def);
Spectrum param_spectrum(lua_State* l, int p, const char* name);
Spectrum param_spectrum_opt(lua_State* l, int p, const char* name, Spectrum def);
Transform param_transform_opt(lua_State* l, int p, const char* name, const Transform& def);
Transform param_transform(lua_State* l, int p, const char* name);
V3 param_vec3(lua_State* l, int p, const char* name, VecKind kind);
void params_check_unused(lua_State* l, int p);
int params_index(lua_State* l, int idx);   // the table at idx (an empty one if none)

// ---- modules ----------------------------------------------------------------------

int open_geometry(lua_State* l);
int open_spectrum(lua_State* l);
int open_shape(lua_State* l);
int open_material(lua_State* l);
int open_light(lua_State* l);
int open_camera(lua_State* l);
int open_builder(lua_State* l);
int open_render(lua_State* l);
int open_image(lua_State* l);
int open_sampler(lua_State* l);
int open_filter(lua_State* l);
int open_chrono(lua_State* l);
int open_stats(lua_State* l);
int open_math(lua_State* l);
int open_env(lua_State* l);
int open_texture(lua_State* l);

// Command-line arguments after the script name (dort.env.get_argv).
void set_argv(std::vector<std::string> argv);

// Record mode: when the environment variable DORT_LUA_RECORD names a file,
// build_scene writes the flat scene there as JSON instead of creating a
// device scene ("%d" in the name is replaced by the scene's number in build
// order), and render_sync produces a black image.  For checking scene
// translation without a GPU.
const char* record_path();
void write_scene_json(const FlatScene& f, const Camera* cam, const char* path);

std::shared_ptr<Image> check_image(lua_State* l, int idx);
void push_image(lua_State* l, std::shared_ptr<Image> img);

}  // namespace dortlua
