/*
 * rmcuda.h - C ABI of the B200 (sm_100a) path-tracing backend for raymotion.
 *
 * This library replaces the reference's Metal backend, whose only entry point
 * is
 *     bool raymotion::render_image_metal(const Scene&, const Camera&,
 *                                        const RenderConfig&, uint64_t seed,
 *                                        std::vector<uint8_t>& rgb,
 *                                        std::string& error);
 * (reference include/raymotion/metal.hpp:6-7, implemented in
 * src/engine/metal.mm:95-414).  The ABI below carries the same information
 * with plain pointers and sizes: the packed fp32 scene that metal.mm builds
 * (metal.mm:109-145, layout of src/engine/metal_types.h:5-30), the camera, the
 * render settings, the seed, and an RGB8 output buffer.  Every function returns
 * RM_OK (0) or a nonzero status and writes a human-readable message into the
 * caller's `err` buffer; nothing throws across the boundary.
 *
 * Threading: a context serialises its calls with a mutex, like the reference's
 * process-wide Context (metal.mm:102-104).  Calls are synchronous unless named
 * *_async.
 */
#ifndef RMCUDA_H
#define RMCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RM_OK 0
#define RM_ERR_INVALID 1      /* bad dimensions, sizes or pointers */
#define RM_ERR_UNAVAILABLE 2  /* no CUDA device, or the device is not sm_100 */
#define RM_ERR_CUDA 3         /* a CUDA call failed; the frame was not completed */
#define RM_ERR_ALLOC 4        /* device or pinned allocation failed */
#define RM_ERR_BVH 5          /* the caller's BVH failed validation */
#define RM_ERR_DEVICE 6       /* a kernel reported an error word (bounded loop ran out) */

typedef struct rm_vec3 { float x, y, z; } rm_vec3;

/* One packed triangle, 176 bytes, field for field the reference's Metal ABI
 * metal_data::Triangle (src/engine/metal_types.h:5-11): scene-space vertices,
 * unnormalised geometric normal n = (v1-v0)x(v2-v0), its normalisation nn,
 * vertex normals, material and texture coordinates.  texture_offset is an index
 * into rm_scene_view.texels or -1. */
typedef struct rm_triangle {
  rm_vec3 v0, v1, v2, n, nn, n0, n1, n2;
  float ar, ag, ab, er, eg, eb, ior, rough, metallic, alpha;
  int32_t shader;
  float tu0, tv0, tu1, tv1, tu2, tv2;
  int32_t texture_offset, texture_width, texture_height;
} rm_triangle;

/* A caller-built binary BVH node: Scene::nodes of the reference
 * (include/raymotion/scene.hpp:57-64, built by src/engine/bvh.cpp:29-248)
 * rounded to fp32.  Internal nodes have count == 0 and children left/right;
 * leaves cover bvh_tri[offset, offset+count). */
typedef struct rm_bvh_node {
  rm_vec3 mn, mx;
  int32_t left, right, offset, count;
} rm_bvh_node;

/* Pinhole camera, the reference's metal_data::Camera (metal_types.h:12-15):
 * position, focal length in pixels, row-major rotation m0..m8. */
typedef struct rm_camera {
  float x, y, z, focal;
  float m0, m1, m2, m3, m4, m5, m6, m7, m8;
} rm_camera;

/* The scene of one frame, as metal.mm uploads it (metal.mm:109-186).
 * nodes == NULL asks the library to build the BVH on the device; nodes != NULL
 * with n_nodes == 0 is an empty BVH on which every ray misses (the reference's
 * params.nodes == 0, pathtrace.metal:121); otherwise nodes/bvh_tri are
 * validated and converted (a caller BVH deeper than 64 levels is rebuilt on
 * the device instead). */
typedef struct rm_scene_view {
  const rm_triangle* tris;
  int32_t n_tris;
  int32_t n_nodes;
  const rm_bvh_node* nodes;
  const int32_t* bvh_tri;   /* n_tris entries when nodes != NULL */
  const int32_t* light_tri; /* emissive triangle indices (Scene::light_tri) */
  const float* light_cdf;   /* running area*luminance sums (Scene::light_cdf) */
  int32_t n_lights;
  float light_total;        /* Scene::light_total */
  const rm_vec3* texels;    /* concatenated linear-RGB textures, top row first */
  int64_t n_texels;
} rm_scene_view;

/* Render settings: raymotion::RenderConfig (include/raymotion/pathtrace.hpp:54-81)
 * in fp32, plus `flags`. */
typedef struct rm_config {
  int32_t width, height, spp, max_bounces;
  float resolution, clamp, adapt_rel, adapt_abs;
  int32_t adapt_min, adapt_step;
  int32_t restir_candidates, restir_spatial;
  float restir_radius;
  int32_t restir_mcap;
  uint32_t flags;
} rm_config;

/* flags.  By default the library reads the reference's environment switches
 * exactly as metal.mm does: UOW2_NOADAPT (:154), UOW2_NOMIS (:157),
 * RAYMOTION_RESTIR=0 (:159), RAYMOTION_RESTIR_CANDIDATES / _SPATIAL (:169-170),
 * RAYMOTION_RESTIR_TEMPORAL=0 (:251-252) and RAYMOTION_DENOISE=0 (:269-271).
 * RM_FLAG_NO_ENV ignores the environment and takes those switches from the
 * flag bits instead. */
#define RM_FLAG_NO_ENV 0x1u
#define RM_FLAG_NOADAPT 0x2u
#define RM_FLAG_NOMIS 0x4u
#define RM_FLAG_RESTIR_OFF 0x8u
#define RM_FLAG_DENOISE_OFF 0x10u
#define RM_FLAG_TEMPORAL_OFF 0x20u
/* Not in the reference (which always applies Russian roulette,
 * pathtrace.metal:715-724, :1246-1250): turn RR off. */
#define RM_FLAG_NO_RR 0x40u
/* Not in the reference: keep temporal ReSTIR / denoise history across frames
 * whose triangles changed (the reference requires an identical scene hash,
 * metal.mm:241-253); geometric rejection still applies per pixel. */
#define RM_FLAG_ANIMATED_HISTORY 0x100u

/* Per-context counters, reset by rmcuda_stats_reset. */
typedef struct rm_stats {
  uint64_t path_samples;    /* (pixel, sample) radiance estimates taken */
  uint64_t rays;            /* traversal queries (closest + any-hit) */
  uint64_t nodes_visited;   /* BVH child-pair records fetched (64 B each) */
  uint64_t tris_tested;     /* Moller-Trumbore tests (48 B records) */
  uint64_t frames;
  uint64_t kernel_launches; /* this library's kernels launched by frame calls */
  uint32_t device_error;    /* last nonzero device error word, 0 if none */
  uint32_t kernel_chain;    /* 1 = render_paths, 8/32 = lane kernels, 2 = ReSTIR chain */
  uint32_t bvh_node_bytes;  /* bytes of one node visit: 80 (8-wide compressed BVH) or 64 (binary) */
  uint32_t bvh_builds;      /* device BVH builds of the resident scene since the context was created */
  uint32_t bvh_refits;      /* device BVH refits of the resident scene since the context was created */
  uint32_t bvh_kept;        /* uploads of the resident scene with unchanged triangles: BVH kept, not rebuilt */
} rm_stats;

typedef struct rmcuda_ctx rmcuda_ctx;

/* Library version string. */
const char* rmcuda_version(void);

/* Create a context on CUDA device `device`.  Returns RM_ERR_UNAVAILABLE with
 * the reference's skip message "Metal backend is not available in this build"
 * when no usable device exists (reference tests/test_metal.cpp:25 treats that
 * string as "skip"). */
int rmcuda_create(rmcuda_ctx** out, int device, char* err, size_t errcap);
void rmcuda_destroy(rmcuda_ctx* ctx);

/* Use the caller's CUDA stream (a cudaStream_t) for all work of this context;
 * NULL restores the context's own stream. */
int rmcuda_set_stream(rmcuda_ctx* ctx, void* cuda_stream, char* err, size_t errcap);

/* One frame, the whole of render_image_metal (metal.mm:95-414): validate, upload
 * the scene, build or convert the BVH, choose the kernel chain (plain or lane
 * path tracer, or ReSTIR generate/spatial/shade + denoise), run it, read back
 * W*H*3 bytes of RGB8 (row-major, top row first) into `rgb` (capacity rgb_cap),
 * keep temporal history.  `hdr`, when not NULL, receives W*H*3 floats of the
 * linear radiance that the tonemap consumed.  Synchronous. */
int rmcuda_render(rmcuda_ctx* ctx, const rm_scene_view* scene, const rm_camera* cam,
                  const rm_config* cfg, uint64_t seed, uint8_t* rgb, size_t rgb_cap,
                  float* hdr, char* err, size_t errcap);

/* Upload a scene and make it the context's resident scene (device BVH built or
 * converted).  Later *_resident calls render it without another upload. */
int rmcuda_scene_upload(rmcuda_ctx* ctx, const rm_scene_view* scene, char* err, size_t errcap);

/* Replace the resident scene's vertices (same triangle count and topology) and
 * refit its BVH on the device; `tris` holds n_tris packed triangles.  After
 * `rebuild_every` refits (0 = never) the BVH is rebuilt instead. */
int rmcuda_scene_update(rmcuda_ctx* ctx, const rm_triangle* tris, int32_t n_tris,
                        int32_t rebuild_every, char* err, size_t errcap);

/* ---- Device-side scene preparation (the reference's Objects runtime,
 * include/raymotion/runtime.hpp:20-146).  A model holds object-space
 * triangles as Objects::init leaves them: the fields of the reference's
 * Triangle that Objects::append reads (fp64).  rmcuda_instances_commit does on
 * the device what Objects::render does on the host before each frame
 * (runtime.hpp:121-131): every model triangle of every instance, in push
 * order, is scaled, rotated about x then y then z, and translated; its vertex
 * normals are divided by the scale, rotated and normalised (runtime.hpp:86-113);
 * the instance's material overrides apply; Scene::add_triangle's precompute,
 * degenerate-triangle rejection and emissive CDF follow (scene.cpp:16-87); the
 * triangles are packed as rm_triangle and become the resident scene.  Its BVH
 * is refitted when the instances name the same models in the same order as
 * the previous commit and the commit count is not a multiple of
 * `rebuild_every` (the reference uses 32), else built; the first commit
 * builds. */
typedef struct rm_model_tri {
  double v0[3], v1[3], v2[3], n0[3], n1[3], n2[3];
  double tu0, tv0, tu1, tv1, tu2, tv2;
  double ar, ag, ab, er, eg, eb, metallic, ior, rough, alpha;
  int32_t shader;
  int32_t reserved;
} rm_model_tri; /* 280 bytes */

/* One Objects::push (runtime.hpp:76-84).  The caller passes the rotation's
 * cos_deg / sin_deg (math.hpp:21-22) so that host and device use the same
 * trigonometric values. */
typedef struct rm_instance {
  int32_t model;
  int32_t reserved;
  double position[3];
  double cos_rot[3], sin_rot[3]; /* of rotation.x, .y, .z */
  double scale[3];               /* nonzero */
  double albedo[3], emission[3]; /* a component < 0 keeps the model's */
  double refract, rough, metallic, alpha; /* NaN keeps the model's (an unset std::optional) */
} rm_instance; /* 184 bytes */

/* Upload a model; *model_id receives its handle. */
int rmcuda_model_create(rmcuda_ctx* ctx, const rm_model_tri* tris, int32_t n_tris, int32_t* model_id, char* err,
                        size_t errcap);
/* Replace a model's triangles (same count): a deforming mesh.  The next
 * commit re-derives its instances' world triangles. */
int rmcuda_model_update(rmcuda_ctx* ctx, int32_t model_id, const rm_model_tri* tris, int32_t n_tris, char* err,
                        size_t errcap);
/* Build the world of `n` instances on the device and make it the resident
 * scene (see above).  Enqueued on the context's stream; returns after one
 * small read-back of the world's triangle and light counts. */
int rmcuda_instances_commit(rmcuda_ctx* ctx, const rm_instance* inst, int32_t n, int32_t rebuild_every, char* err,
                            size_t errcap);
/* Read the resident scene back: up to tri_cap packed triangles, up to
 * light_cap light indices and (float) CDF values; counts[0] = triangles,
 * counts[1] = lights; *light_total = the emissive total. */
int rmcuda_scene_read(rmcuda_ctx* ctx, rm_triangle* tris, int32_t tri_cap, int32_t* light_tri, float* light_cdf,
                      int32_t light_cap, int32_t* counts, float* light_total, char* err, size_t errcap);

/* Render the resident scene.  d_rgb / d_hdr are DEVICE pointers (either may be
 * NULL); the work is enqueued on the context stream and not waited for. */
int rmcuda_render_resident_async(rmcuda_ctx* ctx, const rm_camera* cam, const rm_config* cfg,
                                 uint64_t seed, uint8_t* d_rgb, float* d_hdr,
                                 char* err, size_t errcap);

/* Wait for the context stream and check the device error word. */
int rmcuda_sync(rmcuda_ctx* ctx, char* err, size_t errcap);

/* Trace rays against the resident scene.  rays: n records of 7 floats
 * (ox, oy, oz, dx, dy, dz, tmax), device pointer.  any_hit = 0: closest hit,
 * writing tri (original triangle index, -1 for a miss), t, u, v; any_hit = 1:
 * occlusion only (tri = index of some hit or -1).  Outputs are device
 * pointers; t/u/v may be NULL.  Synchronous. */
int rmcuda_trace(rmcuda_ctx* ctx, const float* d_rays, int32_t n, int32_t any_hit,
                 int32_t* d_tri, float* d_t, float* d_u, float* d_v,
                 char* err, size_t errcap);

/* Ray queries that allocate nothing.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory while they run (an engine
 * whose allocator owns the whole GPU, a fixed-budget real-time loop, a stack
 * that forbids runtime allocation).  Builds a BVH over n_tris caller-owned
 * device triangles and answers n_rays device rays exactly like rmcuda_trace,
 * using only the caller's buffers and one fixed device array inside the
 * library (24 MiB, held by every GPU that loads the library until exit), so
 * n_tris is limited to RMCUDA_NOALLOC_MAX_TRIS; larger scenes are rejected
 * with RM_ERR_INVALID.  The array keeps the last call's contents and is
 * shared by all calls: calls that overlap on the GPU race and must be
 * serialised by the caller.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress), so make it before any stream capture.
 * Works on the current device and `cuda_stream` (NULL: the default stream);
 * returns after the queries finish. */
#define RMCUDA_NOALLOC_MAX_TRIS 65536
int rmcuda_trace_noalloc(const rm_triangle* d_tris, int32_t n_tris, const float* d_rays, int32_t n_rays,
                         int32_t any_hit, int32_t* d_tri, float* d_t, float* d_u, float* d_v,
                         void* cuda_stream, char* err, size_t errcap);

/* ---- Preview frame channel (include/raymotion/preview.hpp:8-27).  A frame
 * goes out as the line "RAY1 <w> <h> <frame> <bytes>\n" and its RGB8 bytes,
 * row-major, top row first.  rmcuda_preview_frame writes a host image;
 * rmcuda_preview_last writes the last frame rendered on the context straight
 * from its device RGB8 image (read back through a pinned buffer).  With
 * grant_fd >= 0 the call then reads one byte from it (the reference reads
 * stdin): RM_PREVIEW_DONE when that descriptor is at end of file, the
 * reference's RenderComplete.  A failed write returns RM_ERR_INVALID with
 * "preview channel closed". */
#define RM_PREVIEW_DONE 7
int rmcuda_preview_frame(int32_t fd, const uint8_t* rgb, int32_t width, int32_t height, int32_t frame,
                         int32_t grant_fd, char* err, size_t errcap);
int rmcuda_preview_last(rmcuda_ctx* ctx, int32_t fd, int32_t frame, int32_t grant_fd, char* err, size_t errcap);

/* ---- Scene objects and batched rendering.  No counterpart in the reference,
 * which renders one scene per call (metal.mm:95-414). */
typedef struct rmcuda_scene rmcuda_scene;

/* Upload a scene into device buffers of its own (BVH built or converted as in
 * rmcuda_render), beside the context's resident scene.  Destroy the scenes of
 * a context before the context. */
int rmcuda_scene_create(rmcuda_ctx* ctx, const rm_scene_view* scene, rmcuda_scene** out,
                        char* err, size_t errcap);
void rmcuda_scene_destroy(rmcuda_ctx* ctx, rmcuda_scene* scene);

/* One frame of a scene object with the single-frame policy of rmcuda_render
 * (plain or lane path tracer, or ReSTIR + denoise when the policy picks it),
 * into DEVICE buffers (either may be NULL); enqueued on the context stream and
 * not waited for. */
int rmcuda_render_scene_async(rmcuda_ctx* ctx, const rmcuda_scene* scene, const rm_camera* cam,
                              const rm_config* cfg, uint64_t seed, uint8_t* d_rgb, float* d_hdr,
                              char* err, size_t errcap);

/* One image of a batch.  Output pointers are DEVICE pointers or NULL. */
typedef struct rm_batch_item {
  const rmcuda_scene* scene;
  rm_camera camera;
  rm_config config;
  uint64_t seed;
  uint8_t* d_rgb;   /* W*H*3 RGB8 */
  float* d_hdr;     /* W*H*3 linear radiance */
  uint32_t* d_aux;  /* W*H*2: xor of the pixel's final lane RNG states, samples taken */
} rm_batch_item;

/* Launch settings of batched rendering (rmcuda_batch_tune picks them). */
typedef struct rm_batch_tuning {
  int32_t pool_chunks;  /* path slots in flight, in chunks of 32 lane slots */
  int32_t tile_shape;   /* pixels of a chunk: 0 a row segment, 1 a near-square block */
  int32_t grid_scale;   /* persistent grids: resident blocks per SM x this (1..4) */
  int32_t graph_waves;  /* waves per CUDA graph launch (even, 2..64); 0: no graph */
  int32_t bvh_width;    /* 2: the binary BVH; 8: the 8-wide compressed BVH (collapsed per scene on first use) */
} rm_batch_tuning;

/* Render many images of (possibly different) scenes, views, resolutions,
 * sample counts and depths together in one pool of path slots.  Each image is
 * what the plain single-frame chain gives it: render_paths (K1) or the 8/32
 * lane kernel (K2) of pathtrace.metal:739-815 with the lane rule of
 * metal.mm:390-394, adaptive sampling and clamp, bit for bit equal to
 * rmcuda_render_scene_async with the same inputs (radiance, RGB8, samples
 * and RNG streams).  Items whose policy picks the ReSTIR chain are rejected
 * (set RM_FLAG_RESTIR_OFF, or restir_spatial 0).  Synchronous. */
int rmcuda_render_batch(rmcuda_ctx* ctx, const rm_batch_item* items, int32_t n, char* err, size_t errcap);

/* Time candidate launch settings on the first waves of this batch, keep the
 * fastest for later rmcuda_render_batch calls on this context and return it
 * in `out` (may be NULL).  Leaves partial images in the items' buffers. */
int rmcuda_batch_tune(rmcuda_ctx* ctx, const rm_batch_item* items, int32_t n, rm_batch_tuning* out,
                      char* err, size_t errcap);
/* Progress of the last batch: for each check between graph replays (every
 * graph_waves waves, or 8 without a graph) the live lane slots (queued to
 * start, trace or finish) and the extension rays queued, at most `cap`
 * records (2 ints each) written.  Returns the number of records. */
int rmcuda_batch_log(rmcuda_ctx* ctx, int32_t* out, int32_t cap);
int rmcuda_batch_get_tuning(rmcuda_ctx* ctx, rm_batch_tuning* out);
int rmcuda_batch_set_tuning(rmcuda_ctx* ctx, const rm_batch_tuning* tuning, char* err, size_t errcap);

/* ---- Differentiable rendering.  No counterpart in the reference, whose
 * triangles carry their material inline (metal_types.h:5-11). */

/* The differentiable parameters of a material, in gradient order. */
typedef struct rm_material {
  float albedo[3];
  float rough;
  float emission[3];
  float ior;
} rm_material;
#define RM_MATERIAL_PARAMS 8

/* Give a scene object materials: triangle i takes the parameters of
 * mats[tri_material[i]] (albedo, rough, emission, ior written into the
 * triangle on the device; -1 keeps the triangle's own values).  tri_material
 * (host, n_tris entries) may be NULL after the first call to keep the
 * mapping; n_materials must then stay the same.  light_cdf (host, the scene's
 * n_lights entries) and light_total replace the light-selection table when
 * light_cdf is not NULL (the caller recomputes them from the new emission, as
 * it built them for the scene view).  Synchronous. */
int rmcuda_scene_set_materials(rmcuda_ctx* ctx, rmcuda_scene* scene, const int32_t* tri_material,
                               const rm_material* mats, int32_t n_materials, const float* light_cdf,
                               float light_total, char* err, size_t errcap);

/* Path-replay adjoint of the frame rmcuda_render_scene_async renders for the
 * same arguments: adds dL/dparams into d_grad (DEVICE, n_materials x
 * RM_MATERIAL_PARAMS floats) given d_dL_dimage (DEVICE, W*H*3 floats, the
 * loss gradient with respect to the linear radiance image).  Sampling is held
 * fixed (random decisions, directions, pdfs, MIS weights, the light sample
 * chosen by RIS NEE and its resampling weight, Russian-roulette
 * probabilities); the material-dependent factors of each path are
 * differentiated; each sample is replayed from its random state instead of
 * being stored.  Needs a fixed sample count (adapt_min 0 or RM_FLAG_NOADAPT).
 * The plain chain (single-candidate or RIS NEE) is replayed from the seed.  On
 * the ReSTIR chain the frame's G-buffer, merged reservoirs and denoiser
 * inputs are the checkpoint: call it after rendering that frame on this
 * context (same scene, camera, config and seed); the reservoirs' light
 * samples and weights and the denoiser's G-buffers and history are held, and
 * d_dL_dimage is the gradient with respect to the frame's final (denoised when
 * the denoiser is on) linear image.  Enqueued, not waited for. */
int rmcuda_backward(rmcuda_ctx* ctx, const rmcuda_scene* scene, const rm_camera* cam, const rm_config* cfg,
                    uint64_t seed, const float* d_dL_dimage, float* d_grad, char* err, size_t errcap);

/* Read the last frame's ReSTIR buffers back in the reference record layouts
 * (metal_types.h:32-56): which = 0 G-buffer (76 B/px), 1 initial reservoir,
 * 2 merged reservoir (60 B/px), 3 shaded HDR (12 B/px).  Host pointer. */
int rmcuda_debug_read(rmcuda_ctx* ctx, int32_t which, void* host, size_t cap,
                      char* err, size_t errcap);

/* Drop temporal history (the reference's CacheGuard, metal.mm:105-108). */
int rmcuda_reset_history(rmcuda_ctx* ctx);

int rmcuda_stats_get(rmcuda_ctx* ctx, rm_stats* out);
int rmcuda_stats_reset(rmcuda_ctx* ctx);

/* Per-stage timing with CUDA events recorded on the context stream around
 * every kernel launch of a frame (off by default).  rmcuda_stage_times
 * returns, per RM_STAGE_*, the summed milliseconds and the launch count since
 * the last rmcuda_stats_reset. */
#define RM_STAGE_PLAIN 0     /* render_paths / lane kernels */
#define RM_STAGE_HASH 1      /* scene hash guarding temporal reuse */
#define RM_STAGE_GENERATE 2  /* ReSTIR primary hit + initial reservoir */
#define RM_STAGE_SPATIAL 3   /* ReSTIR temporal + spatial reuse */
#define RM_STAGE_SHADE 4     /* ReSTIR shading, spp indirect paths */
#define RM_STAGE_TEMPORAL 5  /* denoiser temporal pass */
#define RM_STAGE_ATROUS0 6   /* a-trous stride 1 */
#define RM_STAGE_ATROUS1 7   /* a-trous stride 2 + tonemap */
#define RM_STAGE_TONEMAP 8   /* tonemap alone (denoiser off) */
#define RM_STAGE_WF_EXTEND 9 /* wavefront shading: traversal waves (extension rays, and the shadow rays
                                 when one launch traverses both; their counters stay in WF_SHADOW) */
#define RM_STAGE_WF_SHADOW 10 /* wavefront shading: shadow-ray traversal waves */
#define RM_STAGE_WF_SHADE 11 /* wavefront shading: shading waves (incl. the first) */
#define RM_STAGE_BT_START 12  /* batched rendering: tile refill + sample starts */
#define RM_STAGE_BT_EXTEND 13 /* batched rendering: closest-hit traversal */
#define RM_STAGE_BT_SHADOW 14 /* batched rendering: shadow-ray traversal */
#define RM_STAGE_BT_SHADE 15  /* batched rendering: shading */
#define RM_STAGE_BATCH 16     /* batched rendering: a whole rmcuda_render_batch call */
#define RM_STAGE_ADJOINT 17   /* path-replay adjoint (rmcuda_backward) */
#define RM_STAGE_WF_TAIL 18   /* wavefront shading: the last paths (with their traversals' counters) */
#define RM_STAGE_PREP 19      /* rmcuda_instances_commit: world triangles and BVH refit / build */
#define RM_STAGE_COUNT 20
/* level 0: off; 1: one event pair per stage (the wavefront shading loop counts
 * as RM_STAGE_SHADE, a batch as RM_STAGE_BATCH); 2: also every wavefront
 * launch in its own stage (batches then run without CUDA graphs). */
int rmcuda_profile(rmcuda_ctx* ctx, int level);
/* Per-stage device counters since the last reset: n records of
 * {path samples, rays, BVH nodes visited, triangle tests}. */
int rmcuda_stage_counters(rmcuda_ctx* ctx, uint64_t* out, int32_t n);
/* Queue lengths of the last frame's wavefront shading, read every 4 waves:
 * for each read (unfinished paths, extension rays, shadow rays, microseconds
 * from the first read of the frame to this one), at most `cap` records
 * written to `out` (4 ints each); the last record has empty queues (the
 * loop's end, or the end of its tail launch).  Returns the number of records. */
int rmcuda_wave_log(rmcuda_ctx* ctx, int32_t* out, int32_t cap);
int rmcuda_stage_times(rmcuda_ctx* ctx, double* ms, uint64_t* launches, int32_t n);

#ifdef __cplusplus
}
#endif

#endif /* RMCUDA_H */
