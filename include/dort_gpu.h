/* dort_gpu.h -- C ABI of the B200 (sm_100a) path-tracing hot path.
 *
 * A drop-in for the reference renderer's (honzasp/dort) hot path:
 *   - the ray query of the primitive tree: Primitive::intersect /
 *     intersect_p (include/dort/primitive.hpp:26-33) as reached through
 *     Scene::intersect / intersect_p (src/dort/scene.cpp:8-18),
 *     MeshBvhPrimitive (src/dort/mesh_bvh_primitive.cpp:13-45),
 *     Bvh::traverse_elems (src/dort/bvh.cpp:418-469) and
 *     TriangleUv::hit / Triangle::hit_p (src/dort/triangle.cpp:14-46,102-173);
 *   - the "pt" renderer: Renderer::render (include/dort/renderer.hpp:27) as
 *     implemented by PathRenderer (src/dort/path_renderer.cpp:11-206) and
 *     selected by renderer = "pt" in dort.render.make
 *     (src/dort/lua_render.cpp:102-221).
 *
 * Conventions (all entry points):
 *   - Every call returns an int status: DORT_OK (0) or a negative DORT_ERR_*.
 *     dort_gpu_last_error() returns a thread-local message for the last
 *     failing call on the calling thread.  No C++ exception crosses the ABI.
 *   - The caller owns every host array; the library copies what it keeps.
 *     Device memory created by *_create is owned by the handle until the
 *     matching *_destroy.
 *   - Entry points taking host pointers are synchronous.  *_device variants
 *     take device pointers and a cudaStream_t (passed as void*, NULL = the
 *     legacy default stream) and are asynchronous on that stream.
 *   - A scene handle is not thread-safe; callers serialise access to it.
 *
 * Ray layout: 8 floats per ray = (orig.x, orig.y, orig.z, t_min,
 *                                  dir.x,  dir.y,  dir.z,  t_max),
 * the fields of dort::Ray (include/dort/geometry.hpp:172-186).
 */
#ifndef DORT_GPU_H
#define DORT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DORT_GPU_ABI_VERSION 2

enum dort_status {
  DORT_OK = 0,
  DORT_ERR_INVALID = -1,      /* bad argument (null pointer, bad size, NaN vertex, ...) */
  DORT_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  DORT_ERR_OOM = -3,          /* device or host allocation failed */
  DORT_ERR_TIMEOUT = -4,      /* a bounded device-side wait gave up */
  DORT_ERR_UNSUPPORTED = -5,  /* feature not available in this build */
  DORT_ERR_DEVICE = -6        /* a kernel reported an internal error flag */
};

#define DORT_MISS 0xffffffffu

/* Message for the last failing call on this thread ("" if none). */
const char* dort_gpu_last_error(void);

/* ABI version of the loaded library (DORT_GPU_ABI_VERSION). */
int dort_gpu_abi_version(void);

/* ---- materials ------------------------------------------------------------
 * Material kinds and their parameters; each follows one reference material:
 *   LAMBERT    color = albedo                  lambert_material.cpp:5-35
 *   MIRROR     color = albedo                  mirror_material.cpp:5-29
 *   DIELECTRIC color = reflect tint,
 *              color2 = transmit tint,
 *              param[0] = ior (1.5 default)    dielectric_material.cpp:32-116
 *   PHONG      color = diffuse albedo,
 *              color2 = glossy albedo,
 *              param[0] = exponent             phong_material.cpp:6-106
 *   CONDUCTOR  color = normal-incidence reflectance F0 (Schlick),
 *              param[0] = GGX alpha            (no reference counterpart)
 *   OREN_NAYAR color = albedo,
 *              param[0] = sigma (0: Lambert)   oren_nayar_material.cpp:5-72
 * DIELECTRIC also takes param[1] = ior_outside (0: 1.0) and param[2] != 0 for
 * the thin-slab variant (dielectric_material.cpp:59-61,75-80,93-103); a
 * non-positive ior_inside or ior_outside scatters nothing (:108).
 * A material whose colors are all black scatters nothing (the reference adds
 * no BxDF for a black albedo, lambert_material.cpp:29-35).
 */
enum dort_material_kind {
  DORT_MAT_LAMBERT = 0,
  DORT_MAT_MIRROR = 1,
  DORT_MAT_DIELECTRIC = 2,
  DORT_MAT_PHONG = 3,
  DORT_MAT_CONDUCTOR = 4,
  DORT_MAT_OREN_NAYAR = 5
};

typedef struct dort_material {
  uint32_t kind;
  float color[3];
  float color2[3];
  float param[4];
} dort_material;

/* ---- analytic shapes and delta lights ---------------------------------------
 * An analytic shape is a ShapePrimitive (primitive.cpp:28-58) of one of the
 * reference's quadric / box shapes, placed by an affine shape-to-world
 * transform (3x4, row-major: world = M[:, 0:3] * local + M[:, 3]); the shape
 * is intersected in its own space, as the reference does:
 *   SPHERE    param[0] = radius                      sphere_shape.cpp
 *   DISK      param[0] = radius, param[1] = z        disk_shape.cpp
 *   CUBE      [-1, 1]^3                              cube_shape.cpp
 *   CYLINDER  param[0] = radius, param[1..2] = z_min, z_max (no caps)
 *                                                    cylinder_shape.cpp
 * A non-black `emission` makes the shape a DiffuseLight (diffuse_light.cpp),
 * spheres and disks only.  The light samples and weights its shape under
 * its own transform: `to_world`, or `light_to_world` when flags has
 * DORT_SHAPE_LIGHT_TRANSFORM.  The two differ when a script gives the light
 * and its primitive different transforms, as dort.builder.add_diffuse_light
 * does under a non-identity builder transform (builder_ext.lua:38-48 sets the
 * light's transform again on top of the builder's, lua_builder.cpp:227-232).
 *
 * Delta lights (point_light.cpp, directional_light.cpp):
 *   POINT        rgb = intensity, vec = world position
 *   DIRECTIONAL  rgb = radiance,  vec = direction the light travels in
 */
enum dort_shape_kind {
  DORT_SHAPE_SPHERE = 1,
  DORT_SHAPE_DISK = 2,
  DORT_SHAPE_CUBE = 3,
  DORT_SHAPE_CYLINDER = 4
};

#define DORT_SHAPE_LIGHT_TRANSFORM 1u

/* Where the BVH is built (dort_scene_desc.bvh_build). */
enum {
  DORT_BVH_BUILD_DEFAULT = 0,   /* the device, binned SAH */
  DORT_BVH_BUILD_HOST = 1,      /* binned SAH on the host (32 bins, 3 axes) */
  DORT_BVH_BUILD_DEVICE = 2,    /* binned SAH on the device (same bins and costs) */
  DORT_BVH_BUILD_PLOC = 3       /* Morton order + PLOC on the device: fastest build */
};

typedef struct dort_shape {
  uint32_t kind;
  uint32_t material;
  float param[4];
  float to_world[12];
  float emission[3];
  uint32_t flags;
  float light_to_world[12];
} dort_shape;

enum dort_light_kind { DORT_LIGHT_POINT = 1, DORT_LIGHT_DIRECTIONAL = 2 };

typedef struct dort_light {
  uint32_t kind;
  float rgb[3];
  float vec[3];
  uint32_t reserved;
} dort_light;

/* ---- scene ----------------------------------------------------------------
 * A flat scene: the reference's primitive tree (triangles added with
 * add_triangle / add_shape / add_*ply_mesh*, transforms baked into world
 * space) flattened into one triangle array, plus analytic shapes and delta
 * lights.  Hit ids of shapes follow the triangles: shape k is prim
 * tri_count + k.
 *
 *   tri_material  per-triangle material index (NULL: all 0)
 *   tri_emission  per-triangle RGB radiance (NULL: none); every triangle with
 *                 non-black emission is one one-sided diffuse area light, as
 *                 DiffuseLight on a triangle shape (diffuse_light.cpp:40-111),
 *                 emitting to the side of cross(e2, e1) (triangle.cpp:73)
 *   sky_*         background lights: a non-black sky_const[] gives the
 *                 constant InfiniteLight (infinite_light.cpp:5-65); a sky
 *                 image (sky_width x sky_height RGB float, latitude-longitude,
 *                 row 0 = zenith) gives the EnvironmentLight
 *                 (environment_light.cpp:6-158) with radiance scale
 *                 sky_scale (0,0,0 = 1,1,1), up and forward vectors sky_up /
 *                 sky_fwd (0 = +y / +x)
 *   bvh_width     children per BVH node, 2..8 (0: 8)
 *   bvh_build     DORT_BVH_BUILD_HOST: binned-SAH binary tree built on the
 *                 host; DORT_BVH_BUILD_DEVICE (and DEFAULT): the same binned
 *                 SAH on the device; DORT_BVH_BUILD_PLOC: Morton order and
 *                 Parallel Locally-Ordered Clustering on the device (fastest
 *                 build, slower traversal).  All collapse to the same wide
 *                 format; hits do not depend on the choice (closest hit is a
 *                 property of the triangles).
 *   tri_light_verts  for each emissive triangle, the triangle (3 points) its
 *                 light samples and weights, when that differs from the
 *                 primitive: a light and its primitive placed by different
 *                 transforms, as dort.builder.add_diffuse_light makes them
 *                 under a non-identity builder transform (builder_ext.lua:
 *                 38-48, lua_builder.cpp:227-232); the primitive is still
 *                 what rays hit.  Entries of other triangles are ignored.
 */
typedef struct dort_scene_desc {
  uint32_t struct_size;            /* sizeof(dort_scene_desc) */
  const float* verts;              /* vert_count * 3 */
  uint32_t vert_count;
  const uint32_t* tris;            /* tri_count * 3 vertex indices */
  uint32_t tri_count;
  const uint32_t* tri_material;    /* tri_count, or NULL */
  const dort_material* materials;  /* material_count (>= 1 if tri_material) */
  uint32_t material_count;
  const float* tri_emission;       /* tri_count * 3, or NULL */
  const float* sky_rgb;            /* sky_width * sky_height * 3, or NULL */
  uint32_t sky_width;
  uint32_t sky_height;
  float sky_const[3];
  float sky_scale[3];
  float sky_up[3];
  float sky_fwd[3];
  uint32_t bvh_width;
  uint32_t shape_count;
  const dort_shape* shapes;        /* shape_count, or NULL */
  const dort_light* lights;        /* light_count delta lights, or NULL */
  uint32_t light_count;
  uint32_t bvh_build;              /* DORT_BVH_BUILD_* */
  const float* tri_light_verts;    /* tri_count * 9, or NULL: see below */
  uint32_t flags;                  /* DORT_SCENE_* */
  uint32_t reserved[1];
} dort_scene_desc;

/* dort_scene_desc.flags
 * DORT_SCENE_WATERTIGHT: ray/triangle hits by the watertight test of Woop,
 * Benthin and Wald (JCGT 2013) instead of the reference's Moller-Trumbore
 * (triangle.cpp:14-46, 102-134): a ray through an edge or a vertex shared by
 * triangles hits one of them, never slips between them.  Off by default (the
 * reference's arithmetic, bit-exact t / b1 / b2).  Hits away from edges are
 * the same triangles; t, b1, b2 agree to float rounding.  The leaf triangles
 * then store their three vertices; the path tracers use their general
 * instantiation for such scenes. */
#define DORT_SCENE_WATERTIGHT 1u

typedef struct dort_scene dort_scene;

/* Builds the acceleration structure (on the device or the host, bvh_build)
 * and uploads the scene to the current CUDA device.  Replaces the scene build of build_scene
 * (lua_builder.cpp:113-146) and the Bvh constructor (bvh.cpp:9-55). */
int dort_gpu_scene_create(const dort_scene_desc* desc, dort_scene** out_scene);

/* Frees the scene's device memory.  NULL is accepted. */
int dort_gpu_scene_destroy(dort_scene* scene);

/* Scene statistics: out[0] = BVH node count, out[1] = BVH depth,
 * out[2] = triangle count, out[3] = emissive triangle count,
 * out[4] = device bytes held, out[5] = build milliseconds (scene create:
 * host preparation and BVH build), out[6] = how the BVH was built
 * (DORT_BVH_BUILD_HOST / _DEVICE / _PLOC), out[7] = BVH build milliseconds. */
int dort_gpu_scene_stats(const dort_scene* scene, double out[8]);

/* ---- ray casting ----------------------------------------------------------
 * Closest hit (any_hit = 0), replacing MeshBvhPrimitive::intersect
 * (mesh_bvh_primitive.cpp:13-32): out_prim[i] = hit triangle index or
 * DORT_MISS; out_tb[3i..3i+2] = (t, b1, b2) of the hit (untouched on a miss).
 * The triangle test is the reference's Moller-Trumbore arithmetic, rounded
 * identically, so t, b1, b2 are bit-identical to the reference's for the same
 * triangle.  Among hits at exactly equal t the larger triangle index wins.
 *
 * Any hit (any_hit = 1), replacing MeshBvhPrimitive::intersect_p
 * (mesh_bvh_primitive.cpp:34-45): out_prim[i] = 1 if some triangle is hit
 * with t in [t_min, t_max], else 0; out_tb may be NULL.
 *
 * ray_count is at most 2^32 - 2^24 (DORT_ERR_INVALID above).
 *
 * Host-pointer form: rays, out_prim and out_tb are host arrays. */
int dort_gpu_raycast(dort_scene* scene, const float* rays, size_t ray_count,
                     int any_hit, uint32_t* out_prim, float* out_tb);

/* Device-pointer form of dort_gpu_raycast on a caller stream. */
int dort_gpu_raycast_device(dort_scene* scene, const float* d_rays,
                            size_t ray_count, int any_hit, uint32_t* d_prim,
                            float* d_tb, void* stream);

/* Event-timed device ray cast: runs dort_gpu_raycast_device `repeat` times
 * and writes the mean kernel milliseconds per launch (measured with CUDA
 * events on the launch stream). */
int dort_gpu_raycast_timed(dort_scene* scene, const float* d_rays,
                           size_t ray_count, int any_hit, uint32_t* d_prim,
                           float* d_tb, void* stream, int repeat,
                           float* out_ms_per_launch);

/* ---- rendering ------------------------------------------------------------
 * The "pt" renderer: PathRenderer (path_renderer.cpp:11-206) behind
 * Renderer::render (renderer.hpp:27), with the parameters of
 * dort.render.make (lua_render.cpp:102-145).  The film uses the default box
 * filter of radius 0.5 (each sample lands in its own pixel); non-finite or
 * negative samples are dropped as Renderer::iteration_tiled does
 * (renderer.cpp:36-41); a pixel is sum(L) / count of its kept samples
 * (Film::to_image, film.cpp:90-108).  Iteration 0 samples pixel centres,
 * later iterations jitter uniformly (path_renderer.cpp:15-20).
 *
 * Camera: the columns of its camera-to-world transform (origin, and the
 * images of the camera x, y, z axes) and its kind:
 *   PINHOLE    fov in radians              pinhole_camera.cpp:13-31
 *   ORTHO      dimension (image plane width of the longer side)
 *                                          ortho_camera.cpp:13-26,72-93
 *   THIN_LENS  fov, lens_radius, focal_distance
 *                                          thin_lens_camera.cpp:15-33,100-116
 * Every kind has importance / ray pdf = 1, so a sample's value is the
 * path's radiance (path_renderer.cpp:110). */
enum dort_camera_kind {
  DORT_CAMERA_PINHOLE = 0,
  DORT_CAMERA_ORTHO = 1,
  DORT_CAMERA_THIN_LENS = 2
};

typedef struct dort_camera {
  float origin[3];
  float right[3];
  float up[3];
  float forward[3];
  float fov;
  uint32_t kind;
  float lens_radius;
  float focal_distance;
  float dimension;
} dort_camera;

enum dort_direct_strategy { DORT_DIRECT_MIS = 0, DORT_DIRECT_BSDF = 1, DORT_DIRECT_LIGHT = 2 };

/* dort_render_params.renderer: the "pt" renderer (PathRenderer,
 * path_renderer.cpp), the "lt" light tracer (LightRenderer,
 * light_renderer.cpp:13-181: width x height x iterations light paths, each
 * connected to the camera at its first vertex and every non-delta vertex,
 * min / max path length = min_depth / max_depth + 2 as dort.render.make sets
 * them, lua_render.cpp:146-150) or the "bdpt" bidirectional path tracer
 * (BdptRenderer, bdpt_renderer.cpp: a light and a camera walk per pixel
 * sample, every connection weighted by the balance heuristic, t = 1
 * connections splatted unless renderer_flags has DORT_BDPT_NO_T1_PATHS;
 * max_depth <= 13).  only_direct, sample_all_lights and direct_strategy are
 * "pt" parameters. */
enum dort_renderer { DORT_RENDERER_PT = 0, DORT_RENDERER_LT = 1, DORT_RENDERER_BDPT = 2 };

/* dort_render_params.renderer_flags */
#define DORT_BDPT_NO_T1_PATHS 1u   /* bdpt: use_t1_paths = false */
#define DORT_PT_NO_ROULETTE 2u     /* pt: no Russian roulette (paths run to max_depth);
                                      the reference always plays it
                                      (path_renderer.cpp:101-106).  Same expected
                                      image; for derivative checks, where a
                                      roulette decision that flips under a small
                                      parameter change makes a sample jump */
#define DORT_ADJOINT_MEGAKERNEL 4u /* the adjoint's forward and backward
                                      passes as megakernels (one thread per
                                      pixel and slice of samples) instead of
                                      wavefronts (the same estimator; ignored
                                      by the renders) */

typedef struct dort_render_params {
  uint32_t struct_size;        /* sizeof(dort_render_params) */
  uint32_t width, height;      /* x_res, y_res */
  uint32_t iterations;         /* samples per pixel */
  uint32_t min_depth, max_depth;
  uint32_t only_direct;
  uint32_t sample_all_lights;
  uint32_t direct_strategy;    /* dort_direct_strategy */
  uint32_t renderer;           /* dort_renderer */
  uint64_t seed;
  dort_camera camera;
  uint32_t renderer_flags;     /* DORT_BDPT_NO_T1_PATHS */
  uint32_t reserved[7];
} dort_render_params;

/* Renders into out_rgb (host, width * height * 3 floats, row-major, row 0 at
 * the top).  out_stats (optional, 4 doubles): rays traced, samples kept,
 * kernel milliseconds, samples dropped. */
int dort_gpu_render(dort_scene* scene, const dort_render_params* params,
                    float* out_rgb, double* out_stats);

/* Device-pointer form on a caller stream; d_out_rgb is device memory. */
int dort_gpu_render_device(dort_scene* scene, const dort_render_params* params,
                           float* d_out_rgb, void* stream);

/* No reference counterpart.  dort_gpu_render_device for callers that must not
 * allocate GPU memory during a render (a host application that owns every
 * device allocation under a fixed budget, a real-time loop that cannot absorb
 * cudaFree's device synchronisation).  Same kernels and result; the scratch
 * is a fixed 16 MiB array that the library holds on every GPU it is loaded
 * on, so this call allocates nothing.  Images above 1,048,560 pixels are
 * rejected (DORT_ERR_INVALID), and so is a scene that lives on another device
 * than the current one.  All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress) and
 * keeps it; make it before any stream capture, and do not call this entry
 * point on a device after cudaDeviceReset. */
int dort_gpu_render_device_noalloc(dort_scene* scene, const dort_render_params* params,
                                   float* d_out_rgb, void* stream);

/* ---- wavefront ------------------------------------------------------------
 * No single reference counterpart: the same "pt" estimator as dort_gpu_render
 * (same parameters, same random numbers per pixel and sample, so the same
 * paths), executed as a wavefront of generate / extend / shade / shadow
 * stages over device-resident path queues with path regeneration, looped
 * inside one CUDA graph per frame.  With sample_all_lights every path vertex
 * queues the direct-lighting rays of every light (the queues then hold that
 * many entries per path slot). */
typedef struct dort_wavefront_tuning {
  uint32_t struct_size;        /* sizeof(dort_wavefront_tuning) */
  uint32_t queue_capacity;     /* paths in flight, at most 2^28 (0: auto,
                                  up to 2^24 for a frame, 2^22 for a batch;
                                  each path slot holds about 330 bytes of
                                  device memory; more slots, fewer and
                                  fuller waves) */
  uint32_t trace_block;        /* threads per block, trace stages (0: auto) */
  uint32_t shade_block;        /* threads per block, shade stage (0: auto);
                                  a size above what a stage kernel's registers
                                  allow is lowered to that kernel's limit */
  uint32_t sort_rays;          /* 0: auto (off), 1: on, 2: off -- sort each
                                  wave's extension rays by direction octant
                                  and origin cell before tracing them */
  uint32_t max_waves;          /* waves one frame may take (0: automatic, a
                                  bound a correct frame never reaches: every
                                  path slot's share of the samples times
                                  max_depth + 3 waves each).  A frame that
                                  reaches the bound stops; the host-pointer
                                  entry points return DORT_ERR_TIMEOUT and
                                  the device-pointer ones leave the flag for
                                  dort_gpu_batch_stats / out_stats. */
  uint32_t stage_queues;       /* 0: auto (off), 1: on, 2: off -- the shadow
                                  stage stages its queue through bulk copies
                                  into shared memory (cp.async.bulk, one per
                                  warp and batch of 32 entries, overlapping
                                  the previous batch's traversals); blocks of
                                  at most 256 trace threads */
  uint32_t deterministic;      /* 0: auto (off), 1: on, 2: off -- the frame's
                                  sums in a fixed order: every sample's value
                                  is stored apart (16 bytes per pixel and
                                  sample) and the resolve adds them in
                                  sample order, so that the same frame renders
                                  to the same bits (a path's shadow-ray
                                  additions are ordered too unless it has two
                                  in one wave: a background light under the
                                  MIS BSDF strategy, or sample_all_lights) */
} dort_wavefront_tuning;

/* out_stats (optional, 4 doubles): rays traced, samples kept, kernel
 * milliseconds, waves.  tuning may be NULL (automatic). */
int dort_gpu_render_wavefront(dort_scene* scene, const dort_render_params* params,
                              const dort_wavefront_tuning* tuning, float* out_rgb,
                              double* out_stats);

/* Device-pointer form on a caller stream. */
int dort_gpu_render_wavefront_device(dort_scene* scene, const dort_render_params* params,
                                     const dort_wavefront_tuning* tuning, float* d_out_rgb,
                                     void* stream);

/* Batched rendering: many frames -- different scenes, resolutions, spp and
 * depths -- rendered together by one wavefront (one CUDA graph launch): the
 * path queues mix samples of all jobs, so short jobs do not leave the GPU
 * idle.  A batch snapshots each job's scene (which must stay alive and on the
 * current device) and parameters when it is created; it owns its queues,
 * film and images until destroyed. */
typedef struct dort_batch_job {
  dort_scene* scene;
  dort_render_params params;
} dort_batch_job;

typedef struct dort_batch dort_batch;

int dort_gpu_batch_create(const dort_batch_job* jobs, uint32_t job_count,
                          const dort_wavefront_tuning* tuning, dort_batch** out_batch);
/* Renders every job (asynchronous on `stream`). */
int dort_gpu_batch_render(dort_batch* batch, void* stream);
/* Copies job `job`'s image (width * height * 3 floats) to host memory (waits). */
int dort_gpu_batch_image(dort_batch* batch, uint32_t job, float* out_rgb);
/* Device pointer of job `job`'s image inside the batch. */
int dort_gpu_batch_image_device(dort_batch* batch, uint32_t job, const float** out_d_rgb);
/* out[0] = rays traced, out[1] = waves, out[2] = 1 if the wave bound was hit,
 * out[3] = total samples (waits for the last render). */
int dort_gpu_batch_stats(dort_batch* batch, double out[4]);
int dort_gpu_batch_destroy(dort_batch* batch);

/* No reference counterpart.  The wavefront's autotuner: times candidate
 * tunings on the GPU and writes the fastest to out_tuning (struct_size set).
 * Block sizes (trace, shade) of {64, 128, 256} are ranked on a proxy frame
 * (the frame at up to 8 samples per pixel, 2^22 path slots); path-slot
 * capacities 2^22 .. 2^28 on the frame itself, skipping those beyond twice
 * its work or beyond the free device memory (about 340 bytes per slot).
 * Each candidate runs twice, the faster run counts.  budget_ms bounds the
 * search (0: 30 s); when it runs out the best so far wins.  out_stats
 * (optional, 4 doubles): candidates timed, the chosen frame's milliseconds,
 * milliseconds spent, 1 if the budget cut the search short.  The scene's
 * wavefront queues are left at the last candidate's size. */
int dort_gpu_autotune_wavefront(dort_scene* scene, const dort_render_params* params,
                                double budget_ms, dort_wavefront_tuning* out_tuning,
                                double* out_stats);

/* No reference counterpart.  The same for a batch: capacities 2^21 .. 2^24
 * ranked on a proxy batch (every job at an eighth of its samples, at least
 * 4), blocks of 128 (budget_ms 0: 60 s). */
int dort_gpu_autotune_batch(const dort_batch_job* jobs, uint32_t job_count, double budget_ms,
                            dort_wavefront_tuning* out_tuning, double* out_stats);

/* Measurement entry: renders the same frame wave by wave from the host
 * (without the graph) with CUDA events around each stage; out_ms[0..4] =
 * total milliseconds of regen, extend, shade, shadow, neeb; out_ms[5] = waves;
 * out_rays (optional, 4 doubles) = rays traced in total, by the extend stage
 * (closest hit), by the shadow stage (any hit) and by the BSDF-strategy stage
 * (closest hit). */
int dort_gpu_wavefront_stage_times(dort_scene* scene, const dort_render_params* params,
                                   const dort_wavefront_tuning* tuning, double out_ms[6],
                                   double out_rays[4]);

/* ---- adjoint --------------------------------------------------------------
 * No reference counterpart.  Differentiable rendering of the "pt" estimator
 * with respect to per-triangle Lambert albedo and per-triangle emitted
 * radiance, by path replay backpropagation: the backward pass re-traces every
 * sample from its random numbers (nothing is kept between the forward and the
 * backward call), keeping the path's terms in a short per-path log until the
 * sample's value is known; a path with more terms than the log holds is
 * traced a second time instead.
 *
 * tri_albedo (tri_count * 3, or NULL) replaces the albedo of every triangle
 * whose material is Lambert; tri_emission (tri_count * 3, or NULL) replaces
 * the radiance of the scene's emissive triangles (the set of lights is fixed
 * when the scene is created).  Both stay in effect for later renders of the
 * scene until replaced; NULL removes an override.
 *
 * forward:  renders the image with the overrides: the path tracer as
 *           dort_gpu_render_wavefront with deterministic sums (the same
 *           parameters give the same image), or as dort_gpu_render with
 *           DORT_ADJOINT_MEGAKERNEL; the other renderers as dort_gpu_render.
 * backward: given dLoss/dImage (width * height * 3, host), writes
 *           d_albedo[t*3+c] = dLoss/d albedo and d_emission[t*3+c] =
 *           dLoss/d Le (host, tri_count * 3 each; either may be NULL), for
 *           the same parameters and seed as the forward call.
 * loss_l2:  loss = sum (image - target)^2 and its image gradient, on the GPU. */
/* The scene's last backward pass (4 doubles): engine (0: wavefront, 1:
 * megakernel, 2: wavefront whose overflowing samples outnumbered its list,
 * then the megakernel), samples traced a second time because their terms
 * overflowed the wavefront's per-path log, wavefront rays, waves. */
int dort_gpu_adjoint_stats(dort_scene* scene, double* out_stats);

/* Testing aid: the list of samples a wavefront backward pass traces a second
 * time holds at most `entries` samples (a negative value restores the
 * default), so that tests reach the path taken when it fills. */
int dort_gpu_debug_adjoint_list(long long entries);

int dort_gpu_adjoint_forward(dort_scene* scene, const dort_render_params* params,
                             const float* tri_albedo, const float* tri_emission,
                             float* out_image);
int dort_gpu_adjoint_backward(dort_scene* scene, const dort_render_params* params,
                              const float* tri_albedo, const float* tri_emission,
                              const float* dl_dimage, float* d_albedo, float* d_emission);
int dort_gpu_loss_l2(const float* image, const float* target, size_t count,
                     double* out_loss, float* out_grad);

/* ---- diagnostics ----------------------------------------------------------
 * No reference counterpart.  Builds the device scene's wide BVH on the host
 * and runs the device traversal code compiled for the CPU, with the same
 * outputs as dort_gpu_raycast; needs no GPU.  For checking the BVH builder
 * and the traversal logic only -- the device entry points never use it.
 * out_depth (optional) receives the wide BVH depth. */
int dort_gpu_host_check_raycast(const dort_scene_desc* desc, const float* rays,
                                size_t ray_count, int any_hit, uint32_t* out_prim,
                                float* out_tb, uint32_t* out_depth);

/* No reference counterpart.  Runs the device path-sampling code compiled for
 * the CPU over the pixels [row_begin, row_end) of the image (small images
 * only); writes those rows of out_rgb.  The light tracer and the
 * bidirectional tracer (params->renderer = DORT_RENDERER_LT / _BDPT) render
 * whole frames only (rows 0 .. height).  For checking without a GPU. */
int dort_gpu_host_check_render(const dort_scene_desc* desc, const dort_render_params* params,
                               uint32_t row_begin, uint32_t row_end, float* out_rgb);

/* No reference counterpart.  Quality of the scene's BVH: out[0] = surface
 * area cost relative to the root box (each visited child node and each
 * triangle test costs its box's area), out[1] = node count, out[2] = leaf
 * slots, out[3] = depth.  Reads the nodes back from the device. */
int dort_gpu_scene_bvh_cost(const dort_scene* scene, double out[4]);

/* No reference counterpart.  Builds the mesh's BVH on the device (the binned
 * SAH builder, or PLOC when desc->bvh_build is DORT_BVH_BUILD_PLOC), collapses
 * the device's binary tree again with the host code, and compares:
 * out[0] = node bytes that differ, out[1] = leaf-triangle bytes that differ,
 * out[2] = node count, out[3] = 1 if every triangle is in exactly one leaf,
 * out[4] = device build milliseconds, out[5] = SAH levels or PLOC iterations,
 * out[6] = depth, out[7] = surface area cost.  Needs a GPU. */
int dort_gpu_check_device_bvh(const dort_scene_desc* desc, double out[8]);

/* No reference counterpart.  The BxDF code of one material evaluated and
 * sampled for directions in the local shading frame (z = the normal), for
 * checking the formulas and samplers: for i < n, with wo[3i..3i+2] the fixed
 * direction (towards the viewer),
 *   wi (optional): out_f[3i..] = f(wi, wo) (RGB), out_pdf[i] = the density
 *                  of sampling wi given wo;
 *   u (optional):  three uniforms per entry; out_wi[3i..] = the sampled
 *                  direction, out_sf[3i..] = its f, out_spdf[i] = its pdf
 *                  (0: no sample).
 * All arrays are host memory.  on_device = 1 runs the code on the current
 * GPU, 0 the same code compiled for the host.  The renderers never call it. */
int dort_gpu_bsdf_probe(const dort_material* material, size_t n, const float* wo,
                        const float* wi, const float* u, float* out_f, float* out_pdf,
                        float* out_wi, float* out_sf, float* out_spdf, int on_device);

/* No reference counterpart.  Failure injection for tests of the error paths:
 * after this call the library's next `after` allocations succeed and the one
 * after that fails as if memory were exhausted (device and pinned host
 * allocations, and the host-side scene and BVH builders' large allocations);
 * the entry point that made it returns DORT_ERR_OOM, frees what it had
 * allocated, and later calls work normally.  A negative `after` switches
 * injection off.  Process-wide; not for production use. */
int dort_gpu_debug_fail_alloc(long long after);

#ifdef __cplusplus
}
#endif
#endif /* DORT_GPU_H */
