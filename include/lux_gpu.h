/*
 * lux_gpu.h -- C ABI of the B200 LBVH + wavefront path-tracing library (liblux_gpu.so).
 *
 * Every entry point returns an int status (LUX_OK == 0).  On failure the status names
 * the class of error and lux_last_error() returns a thread-local message.  Handles are
 * opaque; the device memory behind a handle is owned by it.
 *
 * Memory: every array argument may point to host memory or to device memory of the
 * context's device; the library inspects each pointer, and device memory of another GPU
 * is rejected with LUX_ERR_INVALID_ARGUMENT.  Device inputs and outputs are
 * stream ordered on the context's stream and the call returns without waiting.  A host
 * input is staged to the device inside the call; a call with any host output waits
 * for its own work before returning (the behaviour of the reference's std::vector
 * API).  One context per host thread, or external locking: a context carries mutable
 * scratch state.
 *
 * Layouts:
 *   triangles  9 floats per triangle: v0.xyz v1.xyz v2.xyz            (geometry/triangle.h:9-11)
 *   aabbs      6 floats per box: min.xyz max.xyz                      (core/aabb.cuh:10-12)
 *   rays       8 floats per ray: origin.xyz t_min direction.xyz t_max  (core/ray.cuh:10-16,
 *              reordered into two 16-byte halves; time is not used by the BVH queries)
 *   pairs      2 int32 per pair (a, b)                                 (bvh/bvh_overlap.cuh:10-13)
 * Primitive ids are the input indices 0..n-1.
 *
 * Reference interfaces replaced (paths relative to the reference's src/):
 *   bvh/gpu_bvh.cuh:50-61, bvh/bvh_overlap.cuh:21-23, integrator/integrator.h:15-22,
 *   integrator/wavefront_pt.cuh:14-28, scene/prepared_scene.h:35-39.
 */
#ifndef LUX_GPU_H
#define LUX_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUX_ABI_VERSION 1

enum lux_status {
    LUX_OK = 0,
    LUX_ERR_INVALID_ARGUMENT = 1,  /* bad size, null handle, unknown enum value */
    LUX_ERR_CUDA = 2,              /* a CUDA runtime call failed */
    LUX_ERR_OUT_OF_MEMORY = 3,     /* device allocation failed */
    LUX_ERR_MISMATCH = 4,          /* refit input does not match the built topology */
    LUX_ERR_DEVICE_CHECK = 5,      /* a kernel's bounded loop or bounds check tripped */
    LUX_ERR_QUEUE_OVERFLOW = 6,    /* a work queue exceeded its capacity */
    LUX_ERR_BUDGET = 7             /* request does not fit the memory budget */
};

enum lux_prim_kind { LUX_PRIM_TRIANGLES = 0, LUX_PRIM_AABBS = 1 };

typedef struct lux_ctx lux_ctx;
typedef struct lux_bvh lux_bvh;

/* ------------------------------------------------------------------ context */

/* Creates a context on `device`.  stream: a cudaStream_t, or NULL for a stream the
 * context creates and owns. */
int lux_ctx_create(lux_ctx** out, int device, void* stream);
int lux_ctx_destroy(lux_ctx* ctx);
/* Re-targets later calls to another cudaStream_t (NULL: the context's own stream). */
int lux_ctx_set_stream(lux_ctx* ctx, void* stream);
/* Waits for all work the context queued. */
int lux_ctx_synchronize(lux_ctx* ctx);
/* Thread-local description of the last failure on this thread ("" if none). */
const char* lux_last_error(void);
int lux_abi_version(void);
/* Number of kernels this context has launched so far (for launch accounting). */
int lux_ctx_launch_count(lux_ctx* ctx, int64_t* count);

/* Tunables (set by the autotuner or the caller; results never depend on them).
 *   LUX_OPT_TRACE_VARIANT  0 auto (4), 1 one thread per ray, 2 persistent warps with
 *                          refill, 3 one thread per ray over 4-wide nodes, 4 persistent
 *                          warps with refill over 4-wide nodes
 *   LUX_OPT_TRACE_BUDGET   traversal steps per refill round of the persistent kernel
 *   LUX_OPT_RENDER_BATCH   paths in flight per wavefront batch (device memory ~200 B each)
 *   LUX_OPT_PATH_BUDGET    traversal steps per refill round of the path tracer's extension and
 *                          shadow kernels (variant 1 uses one thread per path instead)
 *   LUX_OPT_REFILL_BLOCKS  resident 256-thread blocks per SM of those refilling kernels'
 *                          persistent grids (0: as many as fit, else 1..3)
 * Read only (lux_ctx_get_option), the device memory the context holds for reuse:
 *   LUX_OPT_SCRATCH_BYTES  growable scratch of builds and queries
 *   LUX_OPT_STAGING_BYTES  growable staging of host arguments */
enum lux_option {
    LUX_OPT_TRACE_VARIANT = 1,
    LUX_OPT_TRACE_BUDGET = 2,
    LUX_OPT_RENDER_BATCH = 3,
    LUX_OPT_PATH_BUDGET = 4,
    LUX_OPT_SCRATCH_BYTES = 5,
    LUX_OPT_STAGING_BYTES = 6,
    LUX_OPT_REFILL_BLOCKS = 7
};
int lux_ctx_set_option(lux_ctx* ctx, int32_t option, int64_t value);
int lux_ctx_get_option(lux_ctx* ctx, int32_t option, int64_t* value);

/*
 * Autotuner (no reference counterpart): times candidate settings on the caller's own
 * workload, keeps the fastest in the context and reports it.  Tunables never change
 * results.  lux_autotune_trace: LUX_OPT_TRACE_VARIANT x LUX_OPT_TRACE_BUDGET on n
 * closest-hit rays (device pointer, the lux_trace_closest layout) against `bvh`.
 * lux_autotune_render: one thread per path vs refilling lanes x LUX_OPT_PATH_BUDGET x
 * LUX_OPT_RENDER_BATCH (the paths queued per wavefront batch), then, for refilling
 * lanes, LUX_OPT_REFILL_BLOCKS (the persistent grid's blocks per SM), on a probe render
 * of `scene` (use a probe the size of the real renders).  default_ms is the time with
 * the options in effect before tuning.
 */
typedef struct lux_tune_result {
    int32_t trace_variant;
    int32_t budget;
    int64_t render_batch;     /* 0 for ray-query tuning */
    float best_ms;
    float default_ms;
    int32_t candidates;
    int32_t refill_blocks;    /* 0 for ray-query tuning and one thread per path */
} lux_tune_result;
int lux_autotune_trace(lux_ctx* ctx, lux_bvh* bvh, const float* rays, int32_t n,
                       lux_tune_result* out);

/* ------------------------------------------------------------------ film encoding */

/*
 * Encodes a film of per-pixel sums (width * height * 3 floats, host or device) the way
 * the reference's image writers do, into `out` (host or device):
 *   LUX_FILM_PPM8         bytes of write_ppm (film/ppm.h:37-56): sum / spp, Reinhard,
 *                         clamp, gamma 1/2.2, x 255.999 truncated; rows top first
 *   LUX_FILM_PPM8_LINEAR  bytes of write_debug_ppm_linear (film/ppm.h:58-75)
 *   LUX_FILM_PFM          float32 pixels of write_pfm (film/pfm.h:27-40): sum / spp, rows
 *                         bottom first
 * out holds width * height * 3 bytes (PPM) or floats (PFM); headers are the caller's.
 */
enum lux_film_format { LUX_FILM_PPM8 = 0, LUX_FILM_PPM8_LINEAR = 1, LUX_FILM_PFM = 2 };
int lux_film_encode(lux_ctx* ctx, const float* film_sum, int32_t width, int32_t height,
                    int32_t spp, int32_t format, void* out);

/* ------------------------------------------------------------------ LBVH */

/*
 * Builds a linear BVH over n primitives: per-primitive boxes, their union, 30-bit
 * (morton_bits 30) or 63-bit (63) Morton codes of the box centroids normalised to the
 * union, a stable radix sort of the codes, the Karras hierarchy and a bottom-up box
 * pass.  Bit-exact with build_cpu_lbvh_tree (bvh/cpu_lbvh_builder.h:163-259) for 30
 * bits.  Replaces build_gpu_lbvh (bvh/gpu_bvh.cuh:51).  n == 0 yields an empty BVH.
 */
int lux_lbvh_build(lux_ctx* ctx, const float* prims, int32_t n, int32_t kind,
                   int32_t morton_bits, lux_bvh** out);

/*
 * New primitive geometry, same primitive count and order: recomputes leaf and node
 * boxes bottom-up over the existing topology (Morton order is kept, as in
 * refit_gpu_lbvh, bvh/gpu_bvh.cu:597-613).  LUX_ERR_MISMATCH on a count mismatch.
 * Replaces refit_gpu_lbvh (bvh/gpu_bvh.cuh:52).
 */
int lux_lbvh_refit(lux_ctx* ctx, lux_bvh* bvh, const float* prims, int32_t n);

/*
 * Rebuilds `bvh` in place over a new primitive set of the same kind (any count): the
 * handle's device storage is reused when large enough, so a resident BVH can be
 * rebuilt every frame without device allocation.  Same results as lux_lbvh_build.
 */
int lux_lbvh_rebuild(lux_ctx* ctx, lux_bvh* bvh, const float* prims, int32_t n);

int lux_bvh_destroy(lux_bvh* bvh);

/*
 * Attaches triangles (n x 9 floats, input order) to a BVH built from boxes, so that the
 * ray queries accept it: the reference builds from BvhBuildPrimitive boxes and passes
 * the triangles only at query time (intersect_gpu_bvh_stackless, bvh/gpu_bvh.cu:893-915).
 * Results equal those of a BVH built from the triangles when the boxes are the
 * triangles' boxes.
 */
int lux_bvh_attach_triangles(lux_ctx* ctx, lux_bvh* bvh, const float* tris, int32_t n);

/* Primitive count, kind, Morton width and the root box (6 floats, host). */
int lux_bvh_info(lux_ctx* ctx, const lux_bvh* bvh, int32_t* n, int32_t* kind,
                 int32_t* morton_bits, float* root_bounds);

/*
 * Copies the BVH out in the reference's host tree layout (CpuBvhTree,
 * bvh/cpu_bvh.h:15-32; download_bvh_for_validation, bvh/gpu_bvh.cu:615-665): internal
 * node i (0 <= i < n-1) is Karras node i, leaf k is node n-1+k in sorted order.
 * Any output may be NULL.  sorted_codes: n uint64 (30-bit codes widen to 64);
 * sorted_ids: n; node_left/right: 2n-1 (-1 on leaves); node_bounds: (2n-1)*6 floats.
 */
int lux_bvh_download(lux_ctx* ctx, const lux_bvh* bvh, uint64_t* sorted_codes,
                     int32_t* sorted_ids, int32_t* node_left, int32_t* node_right,
                     float* node_bounds);

/*
 * Structure check of a built BVH: sorted ids form a permutation, the root box is the
 * union of the leaf boxes, codes are sorted, every parent link matches its child slot
 * and a traversal from the root reaches every node exactly once.  *valid = 1 or 0; on 0,
 * `message` (capacity bytes, may be NULL) receives the reason.  Returns LUX_OK unless the
 * check itself could not run.  Replaces validate_gpu_bvh_structure
 * (bvh/gpu_bvh.cuh:53; bvh/gpu_bvh.cu:667-829), with the same messages.
 */
int lux_bvh_validate_structure(lux_ctx* ctx, const lux_bvh* bvh, int32_t* valid, char* message,
                               int32_t message_capacity);

/*
 * The structure check, then: the BVH holds each of the n primitives (host or device
 * array, n x 9 floats for triangles, n x 6 for boxes) exactly once, each leaf box within
 * 1e-4 of its primitive's box.  Replaces validate_gpu_bvh_matches_primitives
 * (bvh/gpu_bvh.cuh:54-56; bvh/gpu_bvh.cu:831-891).
 */
int lux_bvh_validate_primitives(lux_ctx* ctx, const lux_bvh* bvh, const float* prims, int32_t n,
                                int32_t* valid, char* message, int32_t message_capacity);

/*
 * No counterpart in the reference.  The Morton half of lux_lbvh_build (primitive boxes,
 * their union, 30- or 63-bit codes, stable radix sort) written into arrays the caller
 * owns, with every temporary in one static device array of LUX_STATIC_SORT_SCRATCH_BYTES
 * that the library holds on each GPU it is loaded on until the process exits.  The call
 * allocates no device memory.  It is meant for callers that cannot allocate: code whose
 * device memory is already promised to a fixed budget (a server that admits work by
 * bytes, where a cudaMalloc could fail or take memory owed to other requests), and
 * per-frame loops that cannot take the device-wide synchronisation that cudaMalloc and
 * cudaFree may bring.
 * prims (n x 9 floats for triangles, n x 6 for boxes), sorted_codes (n uint64; 30-bit
 * codes widen) and sorted_ids (n) are device pointers on the context's device.  The
 * results equal lux_bvh_download's sorted_codes and sorted_ids after lux_lbvh_build of
 * the same input.  n above LUX_STATIC_SORT_MAX_PRIMS is rejected with
 * LUX_ERR_INVALID_ARGUMENT.
 * The first call on a device looks up the array's device address for that device (and,
 * with lazy module loading, may be the call that loads the library's kernels on it, which
 * is when the array's memory is taken).
 * The address is kept for the life of the process, so the library does not support a
 * cudaDeviceReset of that device while it is loaded.  Each call waits for its stream and
 * reports device checks.  All calls on one device share the one array and each call overwrites
 * it: calls whose GPU work overlaps (other streams, contexts or host threads on the same
 * device) race, so the caller must order them.
 */
#define LUX_STATIC_SORT_MAX_PRIMS 1048576
#define LUX_STATIC_SORT_SCRATCH_BYTES 12845312
int lux_lbvh_morton_sort_static(lux_ctx* ctx, const float* prims, int32_t n, int32_t kind,
                                int32_t morton_bits, uint64_t* sorted_codes,
                                int32_t* sorted_ids);

/*
 * Closest hit of each ray against a triangle BVH.  Visits nodes in the reference's
 * stackless order (bvh/bvh_device.cuh:43-90: left child first, strict t < best), so
 * equal-t ties resolve exactly as in the reference; arithmetic is the reference host
 * code's (no multiply-add contraction), so ids and t equal that code's bit for bit.
 * No hit: id -1, t +inf.
 * hit_t may be NULL.  With 1,048,576 or more rays in host memory the rays are copied in
 * four chunks on a second stream of the context, each traced as soon as it lands, and
 * host results return chunk by chunk (same results as one launch; lux_trace_any too).
 * Replaces intersect_gpu_bvh_stackless (bvh/gpu_bvh.cuh:60-62).
 */
int lux_trace_closest(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays,
                      int32_t* hit_id, float* hit_t);

/*
 * Traversal statistics of lux_trace_closest for the same rays, without writing hits:
 * totals[0] += box tests, totals[1] += triangle tests (int64, host or device).  The
 * counts equal the reference's node visits and triangle tests (bvh/bvh_device.cuh:59-87)
 * because the visit order is the same; they define the traversal's algorithmic bytes.
 */
int lux_trace_closest_stats(lux_ctx* ctx, const lux_bvh* bvh, const float* rays,
                            int32_t nrays, int64_t* totals);

/* Any hit (occlusion) in [t_min, t_max]: hit_id receives some hit primitive or -1.
 * Whether a ray is occluded equals whether lux_trace_closest finds a hit. */
int lux_trace_any(lux_ctx* ctx, const lux_bvh* bvh, const float* rays, int32_t nrays,
                  int32_t* hit_id);

/*
 * Box-overlap pairs.  Self: every (a, b), a < b, whose boxes overlap
 * (query_aabb_overlaps_self, bvh/bvh_overlap.cuh:21).  Cross: every (left, right)
 * primitive pair (query_aabb_overlaps_cross, bvh/bvh_overlap.cuh:22-23).  At most
 * max_pairs pairs are written (in no particular order); *found receives the total, so
 * *found > max_pairs means truncated.
 */
int lux_overlap_self(lux_ctx* ctx, const lux_bvh* bvh, int32_t* pairs, int64_t max_pairs,
                     int64_t* found);
int lux_overlap_cross(lux_ctx* ctx, const lux_bvh* left, const lux_bvh* right,
                      int32_t* pairs, int64_t max_pairs, int64_t* found);

/* ------------------------------------------------------------------ scenes and rendering */

typedef struct lux_scene lux_scene;

/* Material (material/material.h:29-40).  type: 0 Lambert, 1 thin Lambert, 2 GGX,
 * 3 dielectric, 4 interface (null), 5 transparent (tinted filter).  emission_source 0
 * is constant emission; 1 (EmissionSourceKind::Image, Material::image_emissive) reads the
 * emission from scene image emission_image (lux_scene_desc.images) at the surface's
 * texture coordinates, nearest texel, wrapped, times emission_scale (the reference's
 * default scale is 1, 1, 1). */
typedef struct lux_material {
    int32_t type;
    float albedo[3];
    float emission[3];
    int32_t emission_two_sided;   /* 0: single sided (EmissionSidedness::SingleSided) */
    float roughness;
    float metallic;
    float eta;
    int32_t emission_source;
    int32_t emission_image;
    float emission_scale[3];
} lux_material;

/* Indexed triangle mesh in object space (scene/scene_data.h:36-44).  normals and uvs
 * may be NULL (all zero, as add_triangle stores them). */
typedef struct lux_mesh_desc {
    const float* vertices;        /* vertex_count * 3 */
    const float* normals;         /* vertex_count * 3 or NULL */
    const float* uvs;             /* vertex_count * 2 or NULL */
    int32_t vertex_count;
    const uint32_t* indices;      /* triangle_count * 3 */
    const int32_t* material_ids;  /* triangle_count */
    int32_t triangle_count;
} lux_mesh_desc;

/* Instance (scene/scene_data.h:46-51): row-major 3x4 object-to-world matrix (the
 * implicit last row is 0 0 0 1) and its inverse; world_to_object all zero asks the
 * library to invert (inverse_affine, core/mat4.cuh:131-160). */
typedef struct lux_instance_desc {
    int32_t mesh;
    int32_t material_override;    /* -1: per-triangle materials */
    float object_to_world[12];
    float world_to_object[12];
} lux_instance_desc;

/* Explicit light (light/light.h:66-79).  kind: 1 point (vec = position, value =
 * intensity), 2 distant (vec = direction to light, value = radiance), 3 uniform
 * infinite (value = radiance), 4 image infinite (image = index into the scene's
 * images, value = scale; add_image_infinite_light, scene/scene_build.h:40-89).
 * Emissive triangles become area lights automatically. */
typedef struct lux_light_desc {
    int32_t kind;
    float vec[3];
    float value[3];
    int32_t image;
} lux_light_desc;

/* Latitude-longitude environment image: width * height RGB texels, row 0 at the +y
 * pole (theta 0), column 0 at phi 0 (the +x axis), phi growing towards +z. */
typedef struct lux_env_image {
    const float* pixels;
    int32_t width, height;
} lux_env_image;

/* Perspective camera (camera/camera.h:29-38). */
typedef struct lux_camera_desc {
    float origin[3], lower_left[3], horizontal[3], vertical[3], lens_u[3], lens_v[3];
    float lens_radius;
} lux_camera_desc;

/* make_perspective_camera (camera/camera.h:96-126) on the host: vertical field of view
 * in degrees, film aspect, lens radius (0: pinhole) and focal distance (<= 0: the
 * look-at distance). */
int lux_camera_perspective(const float origin[3], const float look_at[3], float vfov_degrees,
                           float aspect, float lens_radius, float focal_distance,
                           lux_camera_desc* out);

typedef struct lux_scene_desc {
    const lux_material* materials;
    int32_t material_count;
    const lux_mesh_desc* meshes;
    int32_t mesh_count;
    const lux_instance_desc* instances;
    int32_t instance_count;
    const lux_light_desc* lights;
    int32_t light_count;
    lux_camera_desc camera;
    const lux_env_image* images;
    int32_t image_count;
} lux_scene_desc;

/* RenderSettings (integrator/render_context.h:16-24).  light_sampler
 * (LightSamplerKind, light/light_distribution.h:27-31): 0 uniform, 1 power (the
 * reference default), 2 light tree (`-light-sampler bvh`: area and point lights picked
 * by a walk of a tree over their boxes weighted by power over squared distance, the
 * other lights by power; falls back to power when no light has bounds). */
typedef struct lux_render_request {
    int32_t width, height, spp, max_depth;
    uint64_t seed;
    int32_t frame_index, sample_offset;
    int32_t light_sampler;
} lux_render_request;

/*
 * Uploads a scene: world-space triangle records, one BLAS per mesh and a TLAS over the
 * instances (the LBVH above), materials and the light tables the reference prepares
 * on the host (scene/scene_prepare.h:268-387: area lights in scene-triangle order, then
 * explicit lights, power alias table).  Replaces PreparedScene::prepare_gpu
 * (scene/prepared_scene.h:35-39).
 */
int lux_scene_create(lux_ctx* ctx, const lux_scene_desc* desc, lux_scene** out);
int lux_scene_destroy(lux_scene* scene);

/* Number of scene triangles, area lights and all lights. */
int lux_scene_info(const lux_scene* scene, int32_t* triangles, int32_t* area_lights,
                   int32_t* lights);

/*
 * lux_render with the reference wavefront tracer's debug images (`-debug-aov shadow,ng,ns`
 * with `-gpu`; RenderOutputs / WavefrontDebugViews, integrator/wavefront_debug.cuh and
 * integrator/wavefront_kernels.cu:287-305, 475-482, 586-592).  Each non-null image
 * receives width * height * 3 per-pixel sums over the samples (divide by spp, as
 * write_debug_ppm_linear does):
 *   ng, ns  the camera ray's hit: 0.5 * (normalize(n) + 1) of the geometric normal and
 *           of the shading normal turned to its side; nothing where the ray misses;
 *   shadow  the path's first scattering hit, when it samples a light: (1, 0.5, 0) for an
 *           invalid light sample, (0.5, 0, 1) for an invalid unoccluded estimate, else
 *           the shadow ray's class: (1, 0, 0) light behind the geometric but not the
 *           shading normal; unblocked (0, 0.35, 0.8) after pass-through surfaces, else
 *           (0.03, 0.03, 0.03); blocked by the source's own material within 16 ray
 *           epsilons (1, 1, 0), by a back face of it (0, 0, 1), a front face of it
 *           (0, 1, 1), another material (0, 1, 0).  Mesh boundary edges are not carried,
 *           so the reference's (1, 0, 1) class reads as (0, 0, 1).
 * film_sum is the same film lux_render writes.  The images are summed with atomics, so
 * their last bits may vary between runs.  Host or device arrays.
 */
int lux_render_aovs(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                    float* film_sum, float* shadow, float* ng, float* ns);

/*
 * Path log: one record per surface vertex a path reaches (PathLogRecord,
 * integrator/pathstate.cuh:19-65; filled as the wavefront tracer's evaluate_hit_kernel
 * does, integrator/wavefront_kernels.cu:84-138, 356-558).  Enumerations keep the
 * reference's values: measures 0 none, 1 solid angle, 2 area, 3 discrete; sources
 * 0 none, 1 camera, 2 BSDF, 3 light, 4 guide; BSDF flags 1 diffuse, 2 glossy, 4 delta
 * reflection, 8 delta transmission, 16 transmission; primitive kind 1 triangle.
 */
enum lux_path_log_event {
    LUX_PATH_EVENT_SURFACE_HIT = 1u << 0,
    LUX_PATH_EVENT_EMISSION = 1u << 1,
    LUX_PATH_EVENT_DIRECT_LIGHT_SAMPLED = 1u << 2,
    LUX_PATH_EVENT_DIRECT_LIGHT_VALID = 1u << 3,
    LUX_PATH_EVENT_BSDF_SAMPLED = 1u << 4,
    LUX_PATH_EVENT_TERMINATED = 1u << 5,
    LUX_PATH_EVENT_SPAWNED_RAY = 1u << 6,
    LUX_PATH_EVENT_DELTA = 1u << 7,
    LUX_PATH_EVENT_PASSTHROUGH = 1u << 8
};
enum lux_path_log_termination {
    LUX_PATH_END_NON_SCATTERING = 1u << 0,
    LUX_PATH_END_MAX_DEPTH = 1u << 1,
    LUX_PATH_END_INVALID_BSDF = 1u << 2,
    LUX_PATH_END_RUSSIAN_ROULETTE = 1u << 3,
    LUX_PATH_END_ZERO_THROUGHPUT = 1u << 4
};

typedef struct lux_path_log_record {
    int32_t pixel_index;
    int32_t sample_index;      /* the request's sample_offset plus the sample */
    int32_t depth;             /* scattering bounces before this vertex */
    int32_t triangle_id;       /* scene triangle */
    int32_t instance_id;       /* PrimitiveRef: instance, mesh, local triangle, kind */
    int32_t mesh_id;
    int32_t local_primitive_id;
    int32_t primitive_kind;
    int32_t material_id;
    int32_t vertex;            /* surface vertices of this path before this one */
    float position[3];
    float ng[3];
    float ns[3];               /* shading normal, turned to the geometric normal's side */
    float wo[3];
    float wi[3];
    float throughput_before[3];
    float throughput_after[3];
    float bsdf_pdf;
    float guide_pdf;           /* always 0: no guiding on this path */
    float light_pdf;
    uint8_t bsdf_pdf_measure;
    uint8_t guide_pdf_measure;
    uint8_t light_pdf_measure;
    uint8_t sample_source;
    uint32_t bsdf_flags;
    uint32_t termination_flags;
    uint32_t event_flags;
} lux_path_log_record;

/*
 * lux_render (film_sum as there) that also logs every path's surface vertices
 * (RenderOutputs::set_path_log, integrator/render_context.h:65-85).  records is a HOST
 * array of capacity entries (null when capacity is 0, to count only); *count receives
 * the number of vertices the render reached.  Records come sorted by (sample_index,
 * pixel_index, vertex), one path's vertices in the order it met them (the reference
 * appends in device-atomic order).  A render with more vertices than capacity returns
 * LUX_ERR_QUEUE_OVERFLOW with *count set and records unspecified (the reference
 * throws).  Per path at most max_depth + 1 vertices, so width * height * spp *
 * (max_depth + 1) always suffices.  The records pass through the context's device
 * staging, which keeps capacity * 152 bytes allocated until the context is destroyed
 * (or a larger staged call replaces it): size capacity for the renders logged.
 */
int lux_render_path_log(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                        float* film_sum, lux_path_log_record* records, int64_t capacity,
                        int64_t* count);

/*
 * Light selection as next-event estimation makes it, for validation: for each i, the
 * light that select_u[i] picks at shading position positions[3i..3i+2] with sampler kind
 * light_sampler (0 uniform, 1 power, 2 light tree), in light-table order (area lights in
 * scene-triangle order, then the explicit lights), or -1; the pmf that selection
 * reports; and the light's pmf at that position as MIS evaluates it.  Replaces
 * sample_scene_light and light_pmf (scene/gpu_scene_light_sampler.cuh:9-96).  Host or
 * device arrays; returns when the results are written.
 */
int lux_scene_select_lights(lux_ctx* ctx, const lux_scene* scene, int32_t light_sampler,
                            const float* positions, const float* select_u, int32_t n,
                            int32_t* light_index, float* pmf, float* eval_pmf);

/*
 * New vertex positions for one mesh (same count): world triangles are recomputed and
 * the mesh's BLAS and the TLAS are refit (not rebuilt) for animation between frames.
 * When an instance of the mesh carries emission, the light tables (areas, powers, the
 * power alias table, the light tree) are re-derived as a scene created from the new
 * vertices would hold them.
 */
int lux_scene_update_mesh(lux_ctx* ctx, lux_scene* scene, int32_t mesh, const float* vertices);

/*
 * Wavefront path tracing (WavefrontPathTracer::render, integrator/wavefront_pt.cu:51-84):
 * film_sum receives width*height*3 floats, the per-pixel SUM over spp (Film::pixels,
 * film/film.h:19-21).  Camera rays, closest hits, per-material shading with NEE, MIS and
 * Russian roulette, and shadow rays through pass-through surfaces follow the reference
 * CPU tracer's arithmetic (integrator/cpu_path_tracer.cpp:403-498).
 */
int lux_render(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
               float* film_sum);
/* Autotuner of the path tracer's tunables on a probe render (see lux_autotune_trace). */
int lux_autotune_render(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* probe,
                        lux_tune_result* out);

/* Same paths, but every sample's radiance is written: samples[(pixel*spp + s)*3 + c]
 * (pixel = y*width + x).  For validation against per-sample reference values. */
int lux_render_samples(lux_ctx* ctx, const lux_scene* scene, const lux_render_request* req,
                       float* samples);

/* Rays traced by the last lux_render* on this context: [0] camera + extension rays,
 * [1] shadow-ray segments (each pass-through re-launch counts), host int64[2]. */
int lux_render_ray_counts(lux_ctx* ctx, int64_t* counts);

/* The traversal work of a render, for its roofline: the same render as lux_render (the
 * same film_sum), run by the one-path-per-thread bounce kernels with every walk
 * counted in the reference's visit order (bvh/bvh_device.cuh:43-90 at both levels of
 * scene/gpu_scene_bvh.cuh:44-135; shadow segments walked to their closest hit, as the
 * reference traces them, integrator/wavefront_kernels.cu:28-83).  stats (host
 * int64[5]): [0] camera + extension rays, [1] shadow-ray segments, [2] box tests,
 * [3] triangle tests, [4] instance (TLAS leaf) visits.  Measurement only: slower than
 * lux_render.  No reference counterpart (the reference counts nothing). */
int lux_render_traversal_stats(lux_ctx* ctx, const lux_scene* scene,
                               const lux_render_request* req, float* film_sum,
                               int64_t* stats);

/* ------------------------------------------------------------------ batched / served rendering */

/*
 * A render server keeps scenes resident and renders many requests at once with one
 * persistent path pool: whenever paths finish, their slots are refilled with camera
 * paths of any admitted request (continuous batching at path granularity), so bounces
 * of different depths, requests and scenes share every kernel launch.  Each pool
 * iteration (new paths, extend, shade, shadow, retire) is one CUDA graph launch and
 * never waits for the host.  Films accumulate in 64-bit fixed point (2^-32), which is
 * order-independent: a request's film is bit-identical whether it renders alone or
 * mixed with others.  It differs from lux_render's sample-order float sum by float
 * rounding only.  Requests are admitted in submission order while the device-memory
 * budget (pool + films) allows; a request that could never fit is rejected with
 * LUX_ERR_BUDGET.  The server owns a private context and worker thread; scenes must
 * stay alive until the server is destroyed.  All lux_server_* calls are thread-safe.
 * (No reference counterpart: the reference renders one request at a time,
 * integrator/wavefront_scheduler.cu:73-131.)
 */
typedef struct lux_server lux_server;

typedef struct lux_server_options {
    int64_t pool_paths;            /* paths in flight; 0: 4,194,304 */
    int64_t memory_budget_bytes;   /* pool + request films; 0: 120 GiB */
    int32_t max_requests;          /* requests admitted at once; 0: 256 */
    int32_t path_budget;           /* LUX_OPT_PATH_BUDGET of the server's kernels; 0: 32 */
} lux_server_options;

enum lux_request_state {
    LUX_REQ_QUEUED = 0,
    LUX_REQ_RUNNING = 1,
    LUX_REQ_DONE = 2,
    LUX_REQ_CANCELLED = 3,
    LUX_REQ_FAILED = 4
};

/* scenes: 1 to 64 resident scenes, created on `device`; they must outlive the server. */
int lux_server_create(int device, lux_scene* const* scenes, int32_t scene_count,
                      const lux_server_options* options, lux_server** out);
/* Queues a render of scenes[scene]; film_sum (host or device, width*height*3 floats) is
 * written when the request completes and must stay valid until then. */
int lux_server_submit(lux_server* server, int32_t scene, const lux_render_request* req,
                      float* film_sum, int64_t* request_id);
int lux_server_poll(lux_server* server, int64_t request_id, int32_t* state);
/* Waits up to timeout_us (< 0: forever) for a final state (done, cancelled, failed). */
int lux_server_wait(lux_server* server, int64_t request_id, int64_t timeout_us,
                    int32_t* state);
/* Waits until every submitted request reached a final state. */
int lux_server_wait_all(lux_server* server, int64_t timeout_us);
/* Queued requests are dropped; running ones stop contributing and finish early. */
int lux_server_cancel(lux_server* server, int64_t request_id);
/* New vertex positions for one mesh of one resident scene: applied between pool
 * iterations as a refit (lux_scene_update_mesh), so later paths see the new frame. */
int lux_server_update_mesh(lux_server* server, int32_t scene, int32_t mesh,
                           const float* vertices);
/* Host timestamps (steady clock, ns) of submission, admission and completion. */
int lux_server_request_times(lux_server* server, int64_t request_id, int64_t* times);
/* stats[9]: [0] pool iterations, [1] camera + extension rays, [2] shadow segments,
 * [3] requests completed, [4] requests admitted, [5] refits applied, [6] bytes in use,
 * [7] longest worker pass between admission checks (ns), [8] longest wait for one
 * iteration's results (ns). */
int lux_server_stats(lux_server* server, int64_t* stats);
int lux_server_destroy(lux_server* server);

/*
 * OBJ meshes (host only; replaces load_obj_into_scene, util/obj_loader.h:107-113, for the
 * options the reference's scenes use).  Parses v / vn / vt / f (1-based or negative
 * indices; quads split on the shorter diagonal as the reference's bundled parser does,
 * larger polygons as fans) and usemtl; skips faces with invalid indices, non-finite
 * positions or an area of at most 1e-12 as the reference's loader does; gives every
 * (position, used normal, used texcoord) corner one mesh vertex in first-use order.
 * The caller adds the mesh with an instance whose object_to_world is the returned
 * placement (make_obj_placement_transform, util/obj_loader.cpp:388-423).
 */
enum lux_obj_normal_mode {      /* ObjNormalMode */
    LUX_OBJ_NORMALS_SOURCE = 0, /* vn where given and nonzero, else none (geometric) */
    LUX_OBJ_NORMALS_SMOOTH = 1, /* vn where given, else area-weighted smooth normals */
    LUX_OBJ_NORMALS_FACE = 2    /* none */
};
enum lux_obj_scale_mode { LUX_OBJ_SCALE_NONE = 0, LUX_OBJ_SCALE_MAX_EXTENT = 1,
                          LUX_OBJ_SCALE_X_EXTENT = 2 };
typedef struct lux_obj_options {  /* ObjLoadOptions (util/obj_loader.h:53-68) */
    int32_t normal_mode;
    int32_t reverse_orientation;
    int32_t flip_texcoord_v;
    int32_t scale_mode;           /* ObjPlacementOptions (util/obj_loader.h:35-41) */
    float target_extent;
    int32_t center_xz;
    int32_t ground_to_y;
    float target_y;
    /* usemtl name -> material id.  With bindings every usemtl must be bound, and faces
     * without usemtl take default_material (an error when it is -1).  Without bindings
     * every face takes default_material; the reference appends a Lambert(0.8) material
     * for it, so pass the id that material will get. */
    const char* const* binding_names;
    const int32_t* binding_ids;
    int32_t binding_count;
    int32_t default_material;
} lux_obj_options;
typedef struct lux_obj_mesh {
    int32_t vertex_count, triangle_count;
    float* vertices;           /* 3 per vertex, object space */
    float* normals;            /* 3 per vertex; zero = none */
    float* uvs;                /* 2 per vertex */
    uint32_t* indices;         /* 3 per triangle */
    int32_t* material_ids;     /* per triangle */
    float object_to_world[12]; /* placement, row-major 3x4 */
    float bounds[6];           /* mesh box, object space */
    int32_t skipped_invalid, skipped_nonfinite, skipped_degenerate;
} lux_obj_mesh;
/* Loads path; *out is null (and LUX_OK) when no face survives.  Free with
 * lux_obj_mesh_free. */
int lux_obj_load(const char* path, const lux_obj_options* options, lux_obj_mesh** out);
void lux_obj_mesh_free(lux_obj_mesh* mesh);

#ifdef __cplusplus
}
#endif

#endif /* LUX_GPU_H */
