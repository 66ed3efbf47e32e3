/* psdr.h -- C ABI of the B200 differentiable path tracer (libpsdr_b200.so).
 *
 * Drop-in replacement for the native layer under torch_psdr's Python API
 * (src/python/torch_psdr.py). All buffers are DEVICE pointers owned by the caller
 * (torch tensors in the Python binding) unless stated otherwise; the library owns
 * only its acceleration structures and scratch memory. Every call takes an explicit
 * CUDA stream (cudaStream_t passed as void*) and never synchronises the device,
 * except the few query calls documented as synchronous.
 *
 * Errors: every entry point returns a psdr_status; psdr_last_error() returns a
 * thread-local message for the last failure (replaces the C++ exceptions of
 * src/optix_def.h:9-81 and the Python asserts of torch_psdr.py).
 */
#ifndef PSDR_H_
#define PSDR_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PSDR_API __attribute__((visibility("default")))
#else
#define PSDR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct psdr_scene psdr_scene;
typedef struct psdr_workspace psdr_workspace;
typedef struct psdr_batch psdr_batch;

typedef enum {
  PSDR_OK = 0,
  PSDR_ERR_INVALID_ARG = 1,
  PSDR_ERR_OOM = 2,
  PSDR_ERR_CUDA = 3,
  PSDR_ERR_TIMEOUT = 4,
  PSDR_ERR_NUMERIC = 5,
  PSDR_ERR_UNSUPPORTED = 6 /* a feature combination the library does not implement */
} psdr_status;

enum { PSDR_TEX_NONE = -1, PSDR_TEX_CONSTANT = 0, PSDR_TEX_UV = 1 };
enum { PSDR_MAT_DIFFUSE = 0, PSDR_MAT_DIFFUSE_BSDF = 1 };
enum { PSDR_CAM_PERSPECTIVE = 0, PSDR_CAM_ORTHOGRAPHIC = 1 };
enum { PSDR_LIGHT_AREA = 0, PSDR_LIGHT_ENV = 1, PSDR_LIGHT_SH9 = 2 };
enum { PSDR_EST_REFERENCE = 0, PSDR_EST_UNBIASED = 1 };

/* A texture (texture.h:16-111; torch_psdr.py:209-269 Texture).
 * UV maps are (height, width, channels) row-major with row 0 at the TOP of the
 * image, i.e. the tensor the user passes; the reference flips rows before
 * flattening (torch_psdr.py:250) and the library applies the same flip when it
 * indexes. Constant textures hold `channels` floats. */
typedef struct {
  int32_t kind;     /* PSDR_TEX_* */
  int32_t channels; /* 1 or 3 */
  int32_t height, width;
  const float* data;
} psdr_texture_desc;

/* A triangle mesh with its material (mesh.cc:5-95 TriangleMesh; torch_psdr.py:343-379). */
typedef struct {
  const float* vertices;  int32_t num_vertices; /* (V,3) */
  const int32_t* faces;   int32_t num_faces;    /* (F,3) */
  const float* uvs;       int32_t num_uvs;      /* (T,2) or NULL */
  const int32_t* uv_indices;                    /* (F,3) or NULL */
  int32_t material;                             /* PSDR_MAT_* */
  psdr_texture_desc color;                      /* diffuse reflectance (3 channels) */
  psdr_texture_desc roughness;                  /* DiffuseBsdf only (1 channel) */
  psdr_texture_desc normal;                     /* DiffuseBsdf only, kind NONE if absent */
} psdr_mesh_desc;

/* A light. AREA (emitter.cc:4-14 AreaLight; torch_psdr.py:388-414): a triangle mesh
 * of constant radiance emit (host data). ENV / SH9 (emitter.cc:94-352 EnvLight,
 * SH9Light; torch_psdr.py:417-452): the library builds the reference's 12-triangle box
 * from box_min / box_max, which the caller computes as scene.cc:31-49 does (the box of
 * the camera positions and mesh vertices around its centre, scaled to 1000 times its
 * largest extent); vertices / faces / emit are ignored. ENV emits its cube map (UV3f,
 * the 4 x 3 cross of the reference's box uvs); SH9 emits sum_k sh9[3k + c] Y_k(wi) of
 * the hit's incoming direction wi. At most one ENV / SH9 light, the last of the array. */
typedef struct {
  const float* vertices; int32_t num_vertices;
  const int32_t* faces;  int32_t num_faces;
  float emit[3];
  int32_t type;                  /* PSDR_LIGHT_* */
  psdr_texture_desc cube_map;    /* ENV */
  float sh9[27];                 /* SH9: (9,3) row-major, host data */
  float box_min[3], box_max[3];  /* ENV / SH9 */
} psdr_area_light_desc;

typedef struct {
  const psdr_mesh_desc* meshes;       int32_t num_meshes;
  const psdr_area_light_desc* lights; int32_t num_lights;
} psdr_scene_desc;

/* A camera (camera.h:208-362; psdr.cc:22-37). Host data. For PERSPECTIVE, fov is
 * the vertical field of view in radians; for ORTHOGRAPHIC it is the view width. */
typedef struct {
  int32_t type;
  float look_from[3], look_at[3], up[3];
  float fov;
  int32_t height, width;
} psdr_camera_desc;

/* PathIntegrator::Config (path_integrator.h:8-21; torch_psdr.py:478-536) plus the
 * B200 extensions: estimator, tile_paths (wavefront tile, 0 = 2^20 paths; see
 * psdr_autotune), leaf_size
 * (BVH leaf collapse, 0 = default), terms, spp_pixel_boundary and seed (0 = the
 * reference's sample streams; seed s offsets every stream index by s * 2654435761
 * modulo 2^32).
 *
 * estimator REFERENCE reproduces the reference's renderD tape (its boundary terms use
 * world-space edge measures and per-pixel sample counts, so their scale is not that of
 * the image derivative). UNBIASED is the derivative of the rendered image itself, in
 * the material form of the path integral: the interior term differentiates the path
 * contribution with the area and camera Jacobians of every vertex, and three boundary
 * terms complete it - material crossing the pixel borders (spp_pixel_boundary samples
 * per unit border segment), silhouettes sliding over the background, and shadow
 * boundaries sliding over the receivers of direct light - with raster-space measures.
 * The forward image is the same for both. */
typedef struct {
  int32_t n_pass, spp_interior, enable_light_visable, spp_primary_edge, spp_secondary_edge;
  int32_t max_bounce, mis_light_samples, mis_bsdf_samples;
  int32_t primary_edge_preprocess_rounds, secondary_edge_preprocess_rounds;
  int32_t primary_edge_hypercube_resolution, secondary_edge_hypercube_resolution[3];
  int32_t estimator;
  int32_t tile_paths;
  int32_t leaf_size;
  int32_t terms;  /* gradient terms of psdr_render_bwd: bit 0 interior, bit 1 primary
                     edges, bit 2 direct edges, bit 3 pixel borders (UNBIASED only),
                     bit 5 interpenetration creases (UNBIASED only, perspective views:
                     the curves where two meshes cut into each other), bit 6 indirect
                     shadow boundaries (UNBIASED only, perspective views, max_bounce >= 2:
                     occlusion of light reflected by other surfaces), bit 4 BRDF jumps
                     of DiffuseBsdfMaterial (UNBIASED only); 0 = all of these that
                     apply (bit 4 when the job holds a DiffuseBsdfMaterial mesh) */
  int32_t spp_pixel_boundary; /* UNBIASED: samples per unit pixel-border segment */
  uint64_t seed;
  int32_t trace_queue; /* ABI 5: rays each SM traverses concurrently in the wavefront
                          closest-hit kernel, in units of 128 (the traversal queue depth;
                          1..8, 0 = 8); psdr_autotune picks it. Results do not depend on it. */
  int32_t batch_lanes; /* ABI 6: psdr_batch_* only: concurrent streams ("lanes"), each with
                          its own wavefront workspace, over which a batch spreads the
                          independent parts of its job -- the forward's tiles, and in the
                          backward the interior tiles and every boundary term of every view
                          (1..8, 0 = 4; psdr_render_* run them one after another). Gradients
                          are bitwise the same for every value. */
  int32_t batch_records; /* ABI 6: psdr_batch_* only: the forward keeps the replay records of
                            every interior path (16 B x (1 + D x R + 2 D) + 8 B per path, D =
                            max_bounce, R = light + BSDF samples + 1) and the backward runs the
                            adjoint from them instead of re-tracing the paths. 0 = when they
                            fit in a quarter of the device memory free at psdr_batch_create,
                            1 = always, -1 = never (re-trace, memory O(tile)). Gradients are
                            bitwise the same either way. */
} psdr_config;

/* Gradient outputs of psdr_render_bwd (caller-owned device buffers, fp32).
 * vertices: one buffer per mesh followed by one per light, each (V,3), may be NULL.
 * textures: one per mesh (same shape as its color texture), may be NULL.
 * emit: one (3,) buffer per light, may be NULL. camera_origin: one (3,) per camera.
 * roughness / normal: one per mesh (same shape as a DiffuseBsdfMaterial's roughness
 * and normal textures; ignored for other meshes), may be NULL.
 * light_params: one per light: an ENV light's cube-map gradient (its texture's shape),
 * an SH9 light's (9,3) coefficient gradient; ignored for AREA lights; may be NULL.
 * camera_lens (ABI 5): one (10,) buffer per camera, may be NULL: the derivative with
 * respect to the camera parameters as they enter its basis and projection -- look_from
 * through the view direction [0..2], look_at [3..5], up [6..8], fov [9] (camera.h:7-64,
 * 111-124, 235-258; torch_psdr.py:145-152 makes all four differentiable). camera_origin
 * is the derivative with the basis held fixed, so d/dlook_from = camera_origin +
 * camera_lens[0..2]. UNBIASED estimator: the image derivative (the camera basis and fov
 * move the image content over the pixel grid). REFERENCE estimator: zeros, as the
 * reference's tape has no path from these inputs to the image (the camera ray's direction
 * is not used after the hit, scene.cc:130-137). Perspective cameras only
 * (PSDR_ERR_UNSUPPORTED for an orthographic camera).
 * With accumulate = 0 the outputs are overwritten, otherwise added to. */
typedef struct {
  float** vertices;
  float** textures;
  float** emit;
  float** camera_origin;
  int32_t accumulate;
  float** roughness;
  float** normal;
  float** light_params;
  float** camera_lens;
} psdr_grad_targets;

/* ---------------------------------------------------------------- general */
PSDR_API const char* psdr_last_error(void);
PSDR_API const char* psdr_version(void);
PSDR_API int32_t psdr_abi_version(void);

/* ---------------------------------------------------------------- scene
 * Replaces Scene::Scene (scene.cc:3-104) + SceneOptix ctor / build_accel
 * (scene_optix.cc:10-46, 187-238) + TriangleMesh edge build (mesh.cc:97-204):
 * checks the index buffers (psdr_scene_validate), then flattens the meshes, builds the
 * edge list and the sampling CDFs and an LBVH, all on `stream`. Texture data pointers
 * are borrowed and must outlive the scene. */
PSDR_API psdr_status psdr_scene_create(const psdr_scene_desc* desc, void* stream, psdr_scene** out);
/* Checks the index buffers of a scene description (extension; the reference does not
 * check them): every face index must lie in [0, num_vertices) of its mesh or area light,
 * every uv index in [0, num_uvs). One device reduction per buffer on `stream` and one
 * host read; PSDR_ERR_INVALID_ARG names the first buffer out of range. psdr_scene_create
 * runs the same check before its build gathers through the indices. */
PSDR_API psdr_status psdr_scene_validate(const psdr_scene_desc* desc, void* stream);
PSDR_API psdr_status psdr_scene_destroy(psdr_scene* scene);
/* Rebuild the acceleration structure, triangle attributes and edges after the
 * vertex buffers changed in place (same topology). */
PSDR_API psdr_status psdr_scene_update(psdr_scene* scene, void* stream);
/* Like psdr_scene_update after vertex positions changed (same meshes, same faces), but
 * the BVH keeps the tree of the last full build and only its node boxes are recomputed:
 * cheaper, and the hits are the same; the tree's quality degrades as the geometry moves
 * away from the state it was built for (psdr_scene_update rebuilds it). Replaces the
 * per-iteration Scene reconstruction of the reference (scene.cc:3-104; its OptiX GAS
 * build, scene_optix.cc:187-238) when only positions change. */
PSDR_API psdr_status psdr_scene_refit(psdr_scene* scene, void* stream);
/* BVH leaves of up to leaf_size (1..8) triangles; rebuilds the scene's geometry.
 * Extension (the reference's OptiX build has no such knob); psdr_autotune picks it. */
PSDR_API psdr_status psdr_scene_set_leaf_size(psdr_scene* scene, int32_t leaf_size, void* stream);
/* Synchronous query: [0] triangles, [1] vertices, [2] edges, [3] bvh nodes,
 * [4] lights, [5] objects. */
PSDR_API psdr_status psdr_scene_info(psdr_scene* scene, int64_t* info6);
/* Synchronous: copies the edge list (v0,v1 global vertex ids; 16 floats per edge:
 * p0, p1, out_direction, n_left, n_right, length) into DEVICE buffers of capacity cap. */
PSDR_API psdr_status psdr_scene_edges(psdr_scene* scene, int32_t* v01, float* geo, int64_t cap, int64_t* n_out, void* stream);

/* Closest hit for n rays (device, 8 floats per ray: ox oy oz tmin dx dy dz tmax).
 * Outputs the global triangle id (-1 on miss), OptiX-convention barycentrics
 * (weights of p1, p2) and t. brute_force 1 tests every triangle (the KAT path); 2 runs
 * the resumable traversal of the wavefront closest-hit kernel instead of the one-shot
 * traversal of 0 (both must return brute force's hits). 
 * Replaces SceneOptix::hit (scene_optix.cc:240-277) + device_programs.cu:13-47. */
PSDR_API psdr_status psdr_intersect(psdr_scene* scene, const float* rays, int64_t n, int32_t* tri, float* bary,
                           float* t, int32_t brute_force, void* stream);

/* Synchronous host query (extension, no device work): the raster-to-direction map of a
 * perspective camera that the camera_lens gradient differentiates, M (3x3 row-major,
 * raster coordinates taken from the image centre: the world direction seen at raster
 * point u is proportional to M [u_x - W/2, u_y - H/2, 1]), and P_j = M^-1 dM/dtheta_j for
 * the ten parameters theta = (look_from, look_at, up, fov) (10 x 9 doubles), built as
 * camera.h:7-64 builds the camera basis. Either output may be NULL. */
PSDR_API psdr_status psdr_camera_lens_jacobian(const psdr_camera_desc* cam, double* m9, double* p90);

/* ---------------------------------------------------------------- rendering
 * psdr_render_fwd replaces PathIntegrator::renderC / the forward of renderD
 * (path_integrator.cc:381-414; torch_psdr.py:538-556). images[c] is a device
 * (H,W,3) fp32 buffer per camera. */
PSDR_API psdr_status psdr_workspace_create(psdr_workspace** out);
PSDR_API psdr_status psdr_workspace_destroy(psdr_workspace* ws);
PSDR_API psdr_status psdr_render_fwd(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams, int32_t n_cams,
                            const psdr_config* cfg, float** images, void* stream);
/* Allocation-free variant of psdr_render_fwd for one camera; no counterpart in the
 * reference. For callers that cannot allocate device memory at render time (a host
 * that gives the library a fixed budget up front, a loop that cannot afford
 * cudaMalloc's implicit device synchronisation). The wavefront tiles use one
 * file-scope 32 MiB __device__ array per GPU, held until the process exits; tiles
 * shrink to fit it, so any image size works, but spp_interior must not exceed the
 * tile (about 100k paths with one light and one BSDF sample; larger values return
 * PSDR_ERR_INVALID_ARG). It takes perspective cameras (others return
 * PSDR_ERR_INVALID_ARG), and the device current at the call must be the one the scene
 * was created on (else PSDR_ERR_INVALID_ARG). The first call on a device resolves the
 * array's address (cudaGetSymbolAddress), so make that first call before any stream
 * capture. All calls share the array and it keeps the last call's contents: calls
 * that overlap on the GPU (other streams, other threads) race and must be serialised
 * by the caller. The scene is an input created earlier by psdr_scene_create; image is
 * the (H,W,3) output. */
PSDR_API psdr_status psdr_render_fwd_noalloc(psdr_scene* scene, const psdr_camera_desc* cam, const psdr_config* cfg,
                                             float* image, void* stream);
/* Per-sample interior radiance of one camera ((H*W*spp, 3) device buffer), the
 * values the film averages; used by the parity tests. */
PSDR_API psdr_status psdr_render_samples(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cam,
                                const psdr_config* cfg, float* samples, void* stream);
/* Autotuner (extension; the reference has no tuner): times forward renders of the
 * given cameras for every wavefront tile size in {2^18, 2^19, 2^20, 2^21} paths, BVH
 * leaf size in {1, 2, 4} triangles (the scene's BVH is rebuilt for each) and traversal
 * queue depth in {4, 6, 8} x 128 rays per SM, keeps the fastest leaf size in the scene
 * (later psdr_scene_update calls use it), writes the fastest tile size and queue depth to
 * cfg->tile_paths / cfg->trace_queue and, when non-null, the leaf size and the fastest
 * render time to best_leaf / best_ms. Allocates and synchronises `stream`; results do
 * not depend on any of the choices (hits and films are deterministic). */
PSDR_API psdr_status psdr_autotune(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams,
                                   int32_t n_cams, psdr_config* cfg, int32_t* best_leaf, float* best_ms,
                                   void* stream);
/* Path-replay adjoint of renderD (replaces Wrap2torch.backward + enoki's reverse
 * sweep, torch_psdr.py:48-72): interior term + the boundary terms of the selected
 * estimator. d_images[c] is dLoss/dImage (H,W,3) per camera. */
PSDR_API psdr_status psdr_render_bwd(psdr_scene* scene, psdr_workspace* ws, const psdr_camera_desc* cams, int32_t n_cams,
                            const psdr_config* cfg, const float** d_images, const psdr_grad_targets* grads,
                            void* stream);

/* ---------------------------------------------------------------- batching
 * Many views over one or more scenes in one work list (small views share tiles),
 * recorded into two CUDA graphs on first use and replayed with one launch each
 * (no counterpart in the reference, which renders cameras one by one with a device
 * synchronisation per ray query, path_integrator.cc:381-406).
 * cam_scene[c] selects the scene of camera c. images / d_images / grads are bound
 * at creation and must stay valid; d_images may be NULL for a forward-only batch.
 * grads has one entry per scene; its camera_origin array is indexed by the global
 * camera index. psdr_batch_forward first rebuilds every scene's geometry from its
 * vertex buffers (so vertices changed in place are picked up), then renders;
 * psdr_batch_backward runs the full adjoint. Both need a non-default stream. */
PSDR_API psdr_status psdr_batch_create(psdr_scene* const* scenes, int32_t n_scenes, const psdr_camera_desc* cams,
                              const int32_t* cam_scene, int32_t n_cams, const psdr_config* cfg, float** images,
                              const float** d_images, const psdr_grad_targets* grads, psdr_batch** out);
PSDR_API psdr_status psdr_batch_forward(psdr_batch* batch, void* stream);
PSDR_API psdr_status psdr_batch_backward(psdr_batch* batch, void* stream);
PSDR_API psdr_status psdr_batch_destroy(psdr_batch* batch);

/* ---------------------------------------------------------------- profiling
 * Extension with no counterpart in the reference. When enabled, the library
 * brackets every trace-kernel launch with CUDA events on the launching stream,
 * counts the kernels it launches and the rays it traces. psdr_profile_read
 * synchronises on the recorded events. */
PSDR_API psdr_status psdr_profile_enable(int32_t on);
PSDR_API psdr_status psdr_profile_reset(void);
/* out[0] kernel launches, out[1] trace launches, out[2] rays traced (all since the
 * last reset); *trace_ms = summed duration of the trace launches. */
PSDR_API psdr_status psdr_profile_read(int64_t* out3, double* trace_ms);

#ifdef __cplusplus
}
#endif
#endif /* PSDR_H_ */
