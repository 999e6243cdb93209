/*
 * cavalry_b200 — C ABI for the BVH build and ray-query hot path (sm_100a).
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch types cross
 * this boundary.  Unless stated otherwise, array arguments are DEVICE pointers
 * and work is enqueued on the caller's CUDA stream (`stream`, a cudaStream_t;
 * NULL = legacy default stream) and completes asynchronously.  Functions return
 * a cav_status; none of them calls exit().  A context is not thread-safe;
 * independent contexts may be used from different threads.
 *
 * Reference interfaces replaced (paths inside AmesingFlank/Cavalry):
 *   BVH::build                      BVH/BVH.h:19, BVH/BVH.cu:317-370
 *   BVH::intersect (closest hit)    BVH/BVH.h:23-107  (called via Core/Scene.h:42-51)
 *   BVH::testVisibility (any hit)   BVH/BVH.h:109-189 (called via Core/Scene.h:53-56)
 */
#ifndef CAVALRY_B200_H
#define CAVALRY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cav_status {
    CAV_OK = 0,
    CAV_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, unsupported flag */
    CAV_ERR_CUDA = 2,             /* a CUDA runtime call failed; see cav_last_error */
    CAV_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
    CAV_ERR_TIMEOUT = 4,          /* a bounded device-side wait gave up */
    CAV_ERR_STACK_OVERFLOW = 5,   /* traversal stack depth exceeded (rays flagged) */
    CAV_ERR_NOT_READY = 6,
    CAV_ERR_CANCELLED = 7         /* the job was cancelled (cav_server_cancel) */
} cav_status;

typedef struct cav_ctx cav_ctx;
typedef struct cav_bvh cav_bvh;

/* Context on CUDA device `device` (the device is made current by every call). */
cav_status cav_ctx_create(int device, cav_ctx** out);
cav_status cav_ctx_destroy(cav_ctx* ctx);
/* Human-readable text of the last error recorded on this context ("" if none). */
const char* cav_last_error(const cav_ctx* ctx);
const char* cav_status_string(cav_status s);
/* ABI version: major*10000 + minor*100 + patch. */
int cav_version(void);
/* Synchronises `stream` and reports the device-side error flags raised since the last
 * check, clearing them: CAV_ERR_TIMEOUT for a radix-sort look-back wait that gave up or a
 * ray stopped at the traversal step limit, CAV_ERR_STACK_OVERFLOW for a full traversal
 * stack, CAV_ERR_INVALID_ARGUMENT for a vertex index out of range in a build, CAV_ERR_CUDA
 * for a broken build or treelet invariant.  The reference reports such conditions with
 * device printf only (Utils/GpuCommons.h:13-20). */
cav_status cav_sync_check(cav_ctx* ctx, void* stream);

/* Bounds of the device-side waits of this context (no wait in any kernel is unbounded):
 *   sort_wait_s     : how long a radix-sort tile waits for its predecessors' published
 *                     digit counts before it gives up, and how long the tcgen05 MLP
 *                     forward waits for a layer's tensor-core completion (<= 0: 2 s);
 *   max_trace_steps : node + triangle visits one ray may take before the traversal stops it
 *                     (prim_id -2 / occluded 2) (<= 0: 2^22).
 * Either ends in CAV_ERR_TIMEOUT from cav_sync_check; the context stays usable. */
cav_status cav_ctx_set_limits(cav_ctx* ctx, double sort_wait_s, int64_t max_trace_steps);
/* Failure injection, for testing the error paths without a device fault:
 *   CAV_INJECT_SORT_STALL (count > 0 on, 0 off): the first tile of every radix-sort pass
 *     withholds its digit counts, so the later tiles' bounded look-back waits run out; the
 *     build completes with CAV_ERR_TIMEOUT from cav_sync_check and a tree that is not
 *     meaningful;
 *   CAV_INJECT_ALLOC_FAIL: the count-th next device allocation made for this context (build
 *     arenas and scratch, scene uploads, render path state, server job buffers) fails once,
 *     and the call that made it returns CAV_ERR_OUT_OF_MEMORY (the others succeed);
 *   CAV_INJECT_MLP_STALL (count > 0 on, 0 off): in the tcgen05 MLP forward, each warpgroup
 *     issues no MMA and no commit for its first tile, so its bounded completion wait runs
 *     out; the call ends with CAV_ERR_TIMEOUT from cav_sync_check and outputs that are not
 *     meaningful;
 *   CAV_INJECT_NONE clears them all.  Nothing here faults, traps or hangs the device. */
enum { CAV_INJECT_NONE = 0, CAV_INJECT_SORT_STALL = 1, CAV_INJECT_ALLOC_FAIL = 2, CAV_INJECT_MLP_STALL = 3 };
cav_status cav_ctx_inject(cav_ctx* ctx, int what, int count);

/*
 * LBVH build + treelet restructuring.  Replaces BVH::build (BVH/BVH.cu:317-370).
 *
 * positions : num_vertices*3 floats (x,y,z), device.
 * indices   : num_triangles*3 int32 vertex indices, device.  Triangle i is the
 *             i-th entry of the reference's global triangle list (mesh order, then
 *             triangle index; Core/TriangleMesh.cu:190-195), so leaf primitive ids
 *             equal the reference's.
 * mesh_ids  : num_triangles int32 (Triangle::meshIndex), device, or NULL (all 0).
 *             Used only by cav_trace_any's mesh exclusion.
 * scene_bounds : 6 host floats (min xyz, max xyz) or NULL.  NULL computes the union
 *             of the triangle boxes on the device (the value Core/Scene.cu:131-135
 *             folds on the host).
 * rounds    : treelet restructuring rounds (>= 0; the reference's
 *             --bvh-opt-rounds, Core/Scene.cu:141-146 picks 3 or 10 when it is -1).
 * The call is stream-ordered; the returned handle may be used on `stream` at once.
 * num_triangles must be in [2, 2^30).  Every vertex index must lie in [0, num_vertices):
 * the kernels check each one, read vertex 0 in place of an index out of range (no load
 * leaves `positions`) and flag it, and the next cav_sync_check returns
 * CAV_ERR_INVALID_ARGUMENT; the tree built from such input is not meaningful.
 */
cav_status cav_bvh_build(cav_ctx* ctx, const float* positions, int64_t num_vertices, const int32_t* indices,
                         const int32_t* mesh_ids, int64_t num_triangles, const float* scene_bounds, int rounds,
                         void* stream, cav_bvh** out);
cav_status cav_bvh_free(cav_bvh* bvh);
int64_t cav_bvh_num_triangles(const cav_bvh* bvh);
/* Tree depth (edges from the root to the deepest leaf); synchronises `stream`. */
cav_status cav_bvh_depth(cav_ctx* ctx, const cav_bvh* bvh, void* stream, int32_t* depth);
/* 1 once the tree's compressed 8-wide view (CAV_TRACE_FAST) has been built, else 0. */
int cav_bvh_has_fast_layout(const cav_bvh* bvh);

/*
 * Parity export of the final node array in the reference's BVHNode order
 * (BVH/BVHNode.h:8-21; BVH/BVH.cu:304-315): 2N-1 records of cav_ref_node, node 0
 * the root.  Internal-node prim ranges are unspecified in the reference and are
 * written as -1 here.  HOST output pointer; synchronises `stream`.
 */
typedef struct cav_ref_node {
    float bmin[3];
    float bmax[3];
    int32_t prim_begin, prim_end, left, right, is_leaf;
} cav_ref_node; /* 44 bytes */
cav_status cav_bvh_export_nodes(cav_ctx* ctx, const cav_bvh* bvh, void* stream, cav_ref_node* host_out);

/*
 * Parity export of the build's intermediate stages: Morton codes in triangle order
 * (BVH/BVH.cu:79-92), the sorted codes and the stable sort permutation (the
 * leaves' primitiveIndexBegin after BVH/BVH.cu:335).  Any pointer may be NULL.
 * HOST outputs of num_triangles entries; synchronises `stream`.
 */
cav_status cav_bvh_export_stages(cav_ctx* ctx, const cav_bvh* bvh, void* stream, uint64_t* morton_unsorted,
                                 uint64_t* morton_sorted, int32_t* sorted_prims);

/* Ray record: 8 floats = origin.xyz, tmin, direction.xyz, tmax (32 bytes, 16-aligned). */
typedef struct cav_ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} cav_ray;

/* trace flags */
#define CAV_TRACE_EXACT 0u        /* reference order and pruning (BVH/BVH.h); default */
#define CAV_TRACE_FAST 2u         /* compressed 8-wide traversal of the same tree: identical hit distances,
                                     equal-distance ties may resolve to a different triangle than the reference order */
#define CAV_TRACE_CULL_ON_POP 1u  /* also re-test a popped node against the current hit
                                     distance / distance limit (fewer visits; results can
                                     differ from the reference only at exact-t ties) */
#define CAV_TRACE_REORDER 4u      /* with either mode, for batches of 65,536 rays or more: trace the rays in the
                                     order of a Morton code of their origins (sorted on the device, stream-ordered
                                     scratch of at most 90 bytes per ray), results written back to each ray's own
                                     index; every ray's result is the one of the given order.  Pays on incoherent
                                     batches (random rays: 11 % fewer cycles); camera and path-ordered rays are
                                     coherent already.  A sort whose look-back wait runs out is reported by
                                     cav_sync_check as CAV_ERR_TIMEOUT. */

/*
 * Closest hit, BVH::intersect semantics (BVH/BVH.h:23-107): nearest child first,
 * a child is visited only if its slab distance is >= 0 and < the current hit
 * distance; the first of equal-t hits in that order wins.  tmin is ignored and
 * tmax limits the accepted distance (tmax = +inf reproduces the reference, which
 * has no tmax).  Outputs (device, any may be NULL except prim_id):
 *   prim_id[i] : hit triangle (reference triangle index) or -1; -2 if the traversal
 *                stack (128 entries, i.e. trees up to 128 deep) overflowed for that
 *                ray or the ray reached the step limit (cav_ctx_set_limits);
 *                cav_sync_check then reports CAV_ERR_STACK_OVERFLOW / CAV_ERR_TIMEOUT.
 *   t[i], uv[2i..2i+1] : hit distance and barycentrics (u, v) of that triangle.
 */
cav_status cav_trace_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int32_t* prim_id,
                             float* t, float* uv, uint32_t flags, void* stream);

/*
 * Any hit, BVH::testVisibility semantics (BVH/BVH.h:109-189): triangles whose mesh
 * id equals the ray's source or target mesh are skipped; with a limit a hit counts
 * only if its distance is < limit.  limit: n floats or NULL (no limit);
 * excl_mesh: 2n int32 (source, target; -1 = none) or NULL.  occluded[i] = 1 if
 * blocked, 0 if visible, 2 if the stack overflowed or the step limit was reached.
 */
cav_status cav_trace_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                         const int32_t* excl_mesh, int64_t n, uint8_t* occluded, uint32_t flags, void* stream);

/*
 * Instrumented traversal: runs the closest-hit (any_hit = 0) or any-hit (any_hit = 1)
 * traversal over `rays` with the same semantics and additionally counts node records
 * fetched (host_counts[0]) and triangles tested (host_counts[1]).  Results are
 * discarded; synchronises `stream`.  Used to state the algorithmic bytes per ray.
 */
cav_status cav_trace_stats(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                           const float* limit, const int32_t* excl_mesh, uint32_t flags, void* stream,
                           uint64_t* host_counts);

/*
 * Host-buffer variants: rays/limit/excl and the outputs are HOST pointers (pageable
 * or pinned).  The context stages them through pinned buffers in chunks, overlapping
 * copies with traversal, and returns after the results are on the host.
 */
cav_status cav_trace_closest_host(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n,
                                  int32_t* prim_id, float* t, float* uv, uint32_t flags);
cav_status cav_trace_any_host(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                              const int32_t* excl_mesh, int64_t n, uint8_t* occluded, uint32_t flags);

/*
 * Launch-shape overrides used by the autotuner (0 = built-in default).
 *   block_threads : threads per traversal block (multiple of 32, <= 1024)
 *   blocks_per_sm : resident blocks requested per SM for the persistent grid
 *   batch         : queue chunk: idle lanes (1..32) a warp accumulates before it claims
 *                   that many new rays from the work counter with one atomic
 */
cav_status cav_set_trace_config(cav_ctx* ctx, int block_threads, int blocks_per_sm, int batch);
/*
 * Traversal-stack override of a mode's single-tree launches (the autotuner sets it):
 *   flags      : CAV_TRACE_EXACT or CAV_TRACE_FAST, the mode whose stack is set
 *   stack      : exact mode: 64 (used only where the tree's depth fits) or 128 entries per
 *                lane, 0 = 128; fast mode: 0
 *   smem_stack : entries per lane kept in shared memory (exact: 16 or 0, fast: 8 or 0); the
 *                rest of the stack is in local memory.  Shared entries cost one L1 wavefront
 *                per push or pop whatever the lanes' depths, and leave less L1 for node data.
 * Results do not depend on either choice.
 */
cav_status cav_set_trace_stack(cav_ctx* ctx, uint32_t flags, int stack, int smem_stack);

/*
 * Allocation-free Morton codes + stable sort (the first stages of BVH::build,
 * BVH/BVH.cu:79-92 and :335) for callers that cannot call cudaMalloc: a renderer
 * embedded in a host application that owns all device memory through a pool fixed at
 * start-up, or a per-frame loop that must neither block on an allocation nor risk one
 * failing mid-frame.  No counterpart in the reference (its build allocates every array
 * it uses).
 *
 * Writes the sorted 63-bit codes to `sorted_codes` and the triangle of each sorted
 * position to `sorted_prims` (device buffers of num_triangles entries, the values
 * cav_bvh_export_stages reports).  positions / indices / scene_bounds as for
 * cav_bvh_build; runs on the current CUDA device and synchronises `stream` before it
 * returns.  Scratch is a static device array sized for CAV_NOALLOC_MAX_TRIANGLES
 * triangles, held by every GPU that loads this library until the process exits; sizes
 * outside [2, CAV_NOALLOC_MAX_TRIANGLES] return CAV_ERR_INVALID_ARGUMENT.  The first call
 * on a device looks up the array's device address and the device's SM count; make that
 * call before any stream capture.  All calls share the array: calls that overlap on the
 * GPU (on different streams or threads) race and must be serialised by the caller.
 * Returns CAV_ERR_INVALID_ARGUMENT for a vertex index outside [0, num_vertices) (the
 * outputs are then not meaningful), CAV_ERR_TIMEOUT when the sort's look-back wait gave
 * up, and CAV_ERR_CUDA for a failed CUDA call or a broken sort invariant.
 */
#define CAV_NOALLOC_MAX_TRIANGLES 131072
cav_status cav_morton_sort_noalloc(const float* positions, int64_t num_vertices, const int32_t* indices,
                                   int64_t num_triangles, const float* scene_bounds, uint64_t* sorted_codes,
                                   int32_t* sorted_prims, void* stream);

/*
 * Scenes and rendering: the reference's Integrator::render (Integrators/PathTracingIntegrator.cu
 * :318-425) over a scene loaded from a .pbrt file by the host parser (SceneLoading/Lexing.cu,
 * SceneLoading/Parsing.cu), behind the CLI surface of main.cu:25-96.
 */
typedef struct cav_scene cav_scene;

typedef struct cav_scene_info_t {
    int width, height, spp, max_depth;
    int64_t triangles;
    int meshes, lights, bvh_rounds;
    int integrator; /* 0 = path, 1 = rlpath, 3 = directlighting */
} cav_scene_info_t;

typedef struct cav_render_opts {
    int spp;                     /* <= 0: the scene's Sampler "pixelsamples" */
    int max_depth;               /* <= 0: the scene's Integrator "maxdepth" */
    int integrator;              /* 0: the scene's Integrator ("path", "rlpath" or "directlighting");
                                    -1: path; 1: rlpath; 2: MLP-guided path (cav_render_guided with
                                    defaults); 3: direct lighting (emission + one light sample per
                                    camera ray, no MIS, as DirectLightingIntegrator.cu) */
    int64_t max_paths_in_flight; /* <= 0: 4M; samples are rendered in chunks of this many paths */
    int width, height;           /* <= 0: the scene's Film resolution (the camera keeps its fov) */
    int flags;                   /* CAV_RENDER_GRAPH: capture one chunk's bounce chain as a CUDA graph and
                                    replay it per chunk, with queue sizes kept on the device (no host round
                                    trip per bounce; path integrator; per-stage times not recorded) */
    int64_t sample_begin;        /* camera samples [sample_begin, sample_end) of the render, numbered
                                    pixel-major (pixel * spp + s, the Halton index); sample_end <= 0: to the
                                    last.  A sub-range renders exactly those samples' contributions, so
                                    films of disjoint ranges sum to the whole render's (path and direct
                                    integrators; a shard of a multi-GPU render) */
    int64_t sample_end;
} cav_render_opts;
enum { CAV_RENDER_GRAPH = 1, CAV_RENDER_FAST_TRACE = 2 /* trace with CAV_TRACE_FAST (path integrator) */ };

/* Host-only .pbrt parse (no GPU): scene counts and the camera-to-world matrix (16 floats,
 * column-major; may be NULL).  On a parse error returns CAV_ERR_INVALID_ARGUMENT and copies the
 * message into err (may be NULL).  bvh_rounds in `info` is reported as -1. */
cav_status cav_pbrt_parse_info(const char* path, int spp_override, const char* integrator_override,
                               cav_scene_info_t* info, float* camera_to_world16, char* err, int err_len);
/* Host-only .pbrt parse to flat triangle arrays (no GPU): world-space positions (3 floats per
 * vertex, meshes concatenated in file order), triangle vertex indices (3 per triangle, global)
 * and the mesh id of every triangle; trianglemesh / plymesh (PLY read from the file beside the
 * .pbrt), sphere and disk shapes as the reference tessellates them.  Call with NULL arrays to
 * get the counts; arrays smaller than the counts give CAV_ERR_INVALID_ARGUMENT.  Parse errors
 * as cav_pbrt_parse_info. */
/* Host-only: decode a texture image exactly as scene loading does (Core/Texture.cu:27-83):
 * 8-bit RGBA, rows bottom-up (flipped on load), colour channels of a .png through the inverse
 * sRGB curve and truncated to 8 bits, alpha unchanged.  PNG only (greyscale, grey + alpha,
 * RGB, RGBA, palette; 8 or 16 bits; not interlaced; at most 32768 texels per side).  With
 * rgba null only width and height are returned; otherwise capacity_bytes must hold
 * 4 * width * height bytes. */
cav_status cav_load_texture_png(const char* path, uint8_t* rgba, int64_t capacity_bytes, int* width, int* height,
                                char* err, int err_len);
/* Host-only: decode an OpenEXR texture exactly as scene loading does for a file name ending in
 * "exr" (Core/Texture.cu:34-57, tinyexr's LoadEXR): RGBA floats, rows in the file's order (no
 * flip, no gamma); R, G, B and A looked up among the first four channels (layer prefixes
 * dropped), a missing A reads 1, a single channel fills all four.  Scanline images with NONE,
 * RLE, ZIPS or ZIP compression and HALF or FLOAT channels; tiled and multi-part files, UINT
 * channels and the PIZ / PXR24 / B44 / DWA codecs are refused (CAV_ERR_INVALID_ARGUMENT, the
 * reason in err), as is a data window of more than 2^28 pixels.  With rgba null only width
 * and height are returned; otherwise capacity_floats must hold 4 * width * height floats. */
cav_status cav_load_texture_exr(const char* path, float* rgba, int64_t capacity_floats, int* width, int* height,
                                char* err, int err_len);
cav_status cav_pbrt_load_triangles(const char* path, float* positions, int64_t max_vertices, int32_t* indices,
                                   int32_t* mesh_ids, int64_t max_triangles, int64_t* num_vertices,
                                   int64_t* num_triangles, char* err, int err_len);
/* Loads a .pbrt scene and builds its BVH.  spp_override > 0 replaces the sampler's
 * pixelsamples (--spp), integrator_override (or NULL) the integrator name (--integrator),
 * bvh_rounds the treelet rounds (--bvh-opt-rounds; -1 = 3, or 10 when spp >= 64, as
 * Core/Scene.cu:141-146).  Parse errors: CAV_ERR_INVALID_ARGUMENT, message in cav_last_error.
 * Synchronous. */
cav_status cav_scene_load_pbrt(cav_ctx* ctx, const char* path, int spp_override, const char* integrator_override,
                               int bvh_rounds, cav_scene** out);
cav_status cav_scene_free(cav_scene* scene);
cav_status cav_scene_info(const cav_scene* scene, cav_scene_info_t* info);
const cav_bvh* cav_scene_bvh(const cav_scene* scene);
/* Renders into a DEVICE film: film_sum (3 floats per pixel) and film_weight (1 per pixel),
 * the reference's Film::samplesSum / samplesWeightSum (Core/Film.h:53-54); pixel = sum / weight.
 * Stream-ordered, except that each bounce reads its queue sizes back to the host. */
cav_status cav_render(cav_ctx* ctx, cav_scene* scene, const cav_render_opts* opts, float* film_sum,
                      float* film_weight, void* stream);
/* Host-film convenience: renders and copies the film to host arrays (3 + 1 floats per pixel);
 * ms_out (or NULL) receives the render time measured with CUDA events. */
cav_status cav_render_to_host(cav_ctx* ctx, cav_scene* scene, const cav_render_opts* opts, float* host_sum,
                              float* host_weight, float* ms_out);
/* Statistics of the scene's last render: paths, closest-hit (extend) and shadow rays traced,
 * bounces, and device time (CUDA events on the render stream) of the whole render and of
 * the extend, shading and shadow stages.  Waits for the render to finish. */
typedef struct cav_render_stats_t {
    int64_t paths, closest_rays, shadow_rays;
    int bounces;
    float ms_total, ms_closest, ms_shade, ms_any;
} cav_render_stats_t;
cav_status cav_render_stats(const cav_scene* scene, cav_render_stats_t* out);
/* Renders the first chunk of paths (opts->max_paths_in_flight, default 4M) and copies the
 * extend-stage rays of bounce `depth` (at most `capacity`) into the DEVICE array rays_out;
 * *count receives how many.  For timing other traversal code on the renderer's own rays.
 * Synchronous. */
cav_status cav_render_capture_rays(cav_ctx* ctx, cav_scene* scene, const cav_render_opts* opts, int depth,
                                   cav_ray* rays_out, int64_t capacity, int64_t* count);
/* Film -> 8-bit sRGB as the reference's Film::readCurrentResult (Core/Film.cu:20-46); HOST arrays. */
cav_status cav_film_to_rgb8(const float* film_sum, const float* film_weight, int width, int height, uint8_t* rgb);
/* Image writers: 8-bit RGB PNG (the reference's output format) and a float PFM of sum/weight. */
cav_status cav_write_png(const char* path, const uint8_t* rgb, int width, int height);
cav_status cav_write_pfm(const char* path, const float* film_sum, const float* film_weight, int width, int height);

/*
 * Serving with continuous batching (serve.cu).  A server owns host threads ("lanes", one by
 * default), each with a stream; jobs are admitted FIFO as the HBM budget and the live-job
 * limit allow, and every tick advances all live jobs of a lane by one bounce with one
 * merged closest-hit and one merged any-hit traversal launch over all their rays (each job
 * against its own resident BVH).  CAV_SERVE_SEQUENTIAL runs one job at a time through the
 * same kernels.  Scenes, BVHs and host buffers must outlive their jobs.
 */
typedef struct cav_server cav_server;
enum { CAV_SERVE_MERGED = 0, CAV_SERVE_SEQUENTIAL = 1 };
enum { CAV_JOB_PENDING = 0, CAV_JOB_RUNNING = 1, CAV_JOB_DONE = 2, CAV_JOB_FAILED = 3, CAV_JOB_CANCELLED = 4 };
typedef struct cav_server_config {
    int64_t hbm_budget_bytes; /* <= 0: 80 GiB */
    int mode;                 /* CAV_SERVE_MERGED or CAV_SERVE_SEQUENTIAL */
    int max_live_jobs;        /* <= 0: 64 */
    int64_t max_paths_per_job; /* path state a render job holds (<= 0: 4M; a job's own
                                  max_paths_in_flight, when set, wins).  Each chunk starts
                                  max(this / live render jobs, min_paths_per_slice) paths */
    uint32_t trace_flags;      /* CAV_TRACE_EXACT (0) or CAV_TRACE_FAST: the merged launches' traversal */
    int lanes;                 /* host threads, each with its own stream and live jobs, ticking
                                  independently on the one GPU (<= 0: 1; sequential mode: 1) */
    int64_t min_paths_per_slice; /* floor of a render job's chunk while others are live (<= 0:
                                  4M, i.e. every chunk as large as the job's state allows);
                                  smaller floors shorten ticks (latency) at some throughput */
    int reject_over_budget;    /* 1: a job whose device memory exceeds the whole budget is refused at
                                  submission (CAV_ERR_OUT_OF_MEMORY); 0: it runs when it is alone */
    int loaders;               /* host threads parsing the scenes of cav_server_submit_scene jobs (<= 0: 4) */
    int64_t graph_max_paths;   /* scene render jobs of at most this many paths run as one graph-replayed
                                  render (every bounce captured, no per-bounce host round trip) instead of
                                  joining the merged ticks (0: 262,144; < 0: never) */
} cav_server_config;
typedef struct cav_job_status {
    int state;         /* CAV_JOB_* */
    cav_status status; /* final status of a finished job */
    double t_submit, t_start, t_done; /* seconds on the server's clock (cav_server_stats.now_s) */
    int64_t bounces;   /* ticks a render job took part in */
} cav_job_status;
typedef struct cav_server_stats_t {
    int64_t ticks, closest_launches, any_launches, max_segments;
    double busy_s, now_s;
    int64_t pending, live, hbm_in_use;
} cav_server_stats_t;
cav_status cav_server_create(cav_ctx* ctx, const cav_server_config* cfg, cav_server** out);
/* Finishes the live jobs, fails the pending ones (CAV_ERR_NOT_READY) and joins the thread. */
cav_status cav_server_destroy(cav_server* server);
/* A render (path integrator) of a loaded scene into HOST films (3 + 1 floats per pixel). */
cav_status cav_server_submit_render(cav_server* server, cav_scene* scene, const cav_render_opts* opts,
                                    float* host_sum, float* host_weight, int64_t* job_id);
/* A job that brings its own scene (a .pbrt file): one of the server's loader threads parses it
 * while the GPU works on other jobs; the job is admitted when its device memory (scene, tree,
 * path state or ray buffers) fits the HBM budget; the admitting lane uploads the scene on its
 * stream and builds its BVH together with those of the other scenes admitted in the same
 * round (one launch per LBVH stage, as cav_bvh_build_batch); the job runs; its scene is
 * released when it ends.  kind CAV_SCENE_RENDER: path integrator into host_sum (3 floats per
 * pixel) and host_weight of render.width x render.height pixels (both required; render.spp and
 * render.max_depth <= 0 take the file's); small renders (config graph_max_paths) are replayed
 * as one CUDA graph.  CAV_SCENE_CLOSEST / CAV_SCENE_ANY: ray queries against the scene's tree,
 * with the arguments and semantics of cav_server_submit_rays.  bvh_rounds: treelet rounds (-1:
 * the reference's default, 3, or 10 when the render's spp >= 64; Core/Scene.cu:141-146).
 * A file that does not parse fails the job with CAV_ERR_INVALID_ARGUMENT.  Host buffers must
 * stay valid until the job is done. */
enum { CAV_SCENE_RENDER = 0, CAV_SCENE_CLOSEST = 1, CAV_SCENE_ANY = 2 };
typedef struct cav_scene_job {
    const char* pbrt_path;
    int kind;
    int bvh_rounds;
    cav_render_opts render;
    float* host_sum;
    float* host_weight;
    const cav_ray* host_rays;
    const float* host_limit;
    const int32_t* host_excl;
    int64_t n_rays;
    int32_t* host_prim;
    float* host_t;
    float* host_uv;
    uint8_t* host_occ;
} cav_scene_job;
cav_status cav_server_submit_scene(cav_server* server, const cav_scene_job* job, int64_t* job_id);
/* A ray-query job on HOST arrays: closest hit (prim, t, uv; t/uv may be NULL) or any hit
 * (occ; limit / excl may be NULL), with the semantics of cav_trace_closest / cav_trace_any. */
cav_status cav_server_submit_rays(cav_server* server, const cav_bvh* bvh, int any_hit, const cav_ray* host_rays,
                                  const float* host_limit, const int32_t* host_excl, int64_t n, int32_t* host_prim,
                                  float* host_t, float* host_uv, uint8_t* host_occ, int64_t* job_id);
/* Cancels a job.  A pending job leaves the queue at once; a running job is stopped by its
 * lane before its next bounce, its device state freed, and its host outputs are left as they
 * are (partial).  Either way the job ends in CAV_JOB_CANCELLED and cav_server_wait returns
 * CAV_ERR_CANCELLED; a job that already finished is not changed.  Other jobs are unaffected. */
cav_status cav_server_cancel(cav_server* server, int64_t job_id);
cav_status cav_server_poll(cav_server* server, int64_t job_id, cav_job_status* status);
/* Waits for a job (timeout_s < 0: forever); returns the job's status or CAV_ERR_TIMEOUT. */
cav_status cav_server_wait(cav_server* server, int64_t job_id, double timeout_s, cav_job_status* status);
cav_status cav_server_stats(cav_server* server, cav_server_stats_t* out);

/* Launch-shape autotuner: times the closest-hit (any_hit = 0) or any-hit traversal of a
 * DEVICE ray sample over candidate shapes (64/128/256 threads per block; queue chunk 1-32;
 * a 64-entry traversal stack when the tree's depth allows it, else 128; the stack's first
 * 16 entries in shared memory or all of it in local memory) and installs the fastest in ctx
 * for later single-tree traversals (merged launches always use the full stack in local
 * memory).  ms is the best launch time of the chosen shape on the sample; smem_stack is the
 * number of stack entries per lane the chosen shape keeps in shared memory (exact mode 16 or
 * 0, fast mode 8 or 0). */
typedef struct cav_trace_config_t {
    int block_threads, blocks_per_sm, batch, stack;
    float ms;
    int smem_stack;
} cav_trace_config_t;
cav_status cav_trace_autotune(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                              const float* limit, const int32_t* excl, void* stream, cav_trace_config_t* best);
/* The same search for the traversal mode in flags (CAV_TRACE_EXACT or CAV_TRACE_FAST, with
 * CAV_TRACE_REORDER when the batches will be traced reordered: every candidate then traces
 * the reordered sample); each mode keeps its own tuned shape in ctx (stack is 0 for the
 * fast mode). */
cav_status cav_trace_autotune_flags(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                                    const float* limit, const int32_t* excl, uint32_t flags, void* stream,
                                    cav_trace_config_t* best);

/*
 * Learned directional proposal (mlp.cu): an MLP from a surface point (position in the scene
 * box and normal angles, 5 floats in [0, 1]) to a mixture of 8 von Mises-Fisher lobes (32
 * outputs: per lobe a weight logit, theta = pi sigmoid, phi = 2 pi sigmoid, kappa =
 * softplus + 0.01), trained on weighted directions with the loss mean(-w log q(omega)).
 * Parameters are FP32 (cav_mlp_num_params of them: per layer W[out][in] then b[out], for
 * 160->64, 64->64, 64->64, 64->32 with one-blob inputs); the kernels use BF16 copies with
 * FP32 accumulation.  Arrays are DEVICE unless named host_.
 */
typedef struct cav_mlp cav_mlp;
int cav_mlp_num_params(void);
cav_status cav_mlp_create(cav_ctx* ctx, uint64_t seed, cav_mlp** out);
cav_status cav_mlp_free(cav_mlp* mlp);
cav_status cav_mlp_get_params(cav_mlp* mlp, float* host_params);
cav_status cav_mlp_set_params(cav_mlp* mlp, const float* host_params);
/* Forward-pass kernel of a network (training and inference): CAV_MLP_KERNEL_TCGEN05 (the
 * default: 128-sample tiles on the tcgen05 tensor cores, accumulators in TMEM) or
 * CAV_MLP_KERNEL_MMA_SYNC (16-sample warp tiles with mma.sync, kept for comparison).  Both
 * compute the same BF16-operand, FP32-accumulate products; results agree to FP32
 * accumulation order.  A tcgen05 completion wait that runs out (1 s) is reported by
 * cav_sync_check as CAV_ERR_TIMEOUT. */
enum { CAV_MLP_KERNEL_TCGEN05 = 0, CAV_MLP_KERNEL_MMA_SYNC = 1 };
cav_status cav_mlp_set_kernel(cav_mlp* mlp, int kernel);
/* in: n x 5, out: n x 32 */
cav_status cav_mlp_forward(cav_mlp* mlp, const float* in, int64_t n, float* out, void* stream);
/* Loss gradient w.r.t. every parameter for one batch (in n x 5, dirs n x 3 unit, w n),
 * copied to host_grads (num_params floats) with the batch loss; no update.  Synchronous. */
cav_status cav_mlp_gradients(cav_mlp* mlp, const float* in, const float* dirs, const float* w, int64_t n,
                             float* host_grads, float* host_loss);
/* One Adam step (beta 0.9 / 0.999) on one batch; stream-ordered. */
cav_status cav_mlp_train_step(cav_mlp* mlp, const float* in, const float* dirs, const float* w, int64_t n, float lr,
                              void* stream);
cav_status cav_mlp_last_loss(cav_mlp* mlp, float* loss);
/* Mixture density of dirs (n x 3) under decoded outputs (n x 32) into pdf, and/or samples
 * (n x 3) drawn with u (n x 3 uniforms); either pair may be NULL. */
cav_status cav_mlp_mixture(cav_ctx* ctx, const float* out, int64_t n, const float* dirs, float* pdf, const float* u,
                           float* samples, void* stream);

/* MLP-guided path integrator (guided.cu): the path integrator whose continuation at
 * non-delta surfaces draws, with probability alpha, from the network's mixture instead of
 * the BSDF, weighted by the one-sample mixture density (unbiased for any network); rendered
 * in passes of 1, 1, 2, 4, ... spp with the network trained after every pass but the last
 * on up to train_samples_per_pass vertices (direction, luminance of returned radiance over
 * throughput).  mlp: a network to use and keep training (NULL: a fresh one for this
 * render).  Also reachable as cav_render with integrator 2 (fresh network, defaults). */
typedef struct cav_guide_opts {
    float alpha;                  /* <= 0: 0.5 */
    int64_t train_samples_per_pass; /* <= 0: 2^18 */
    int train_steps_per_pass;     /* <= 0: 32 */
    int train_batch;              /* <= 0: 16384 */
    float learning_rate;          /* <= 0: 3e-3 */
    int freeze;                   /* 1: use the network as is, no training */
    uint64_t seed;                /* network initialisation when mlp is NULL (0: 1) */
} cav_guide_opts;
typedef struct cav_guide_stats {
    int passes;
    int64_t train_samples, train_steps;
    float last_loss;
} cav_guide_stats;
cav_status cav_render_guided(cav_ctx* ctx, cav_scene* scene, const cav_render_opts* opts, cav_mlp* mlp,
                             const cav_guide_opts* gopts, float* film_sum, float* film_weight, void* stream,
                             cav_guide_stats* stats);

/* Builds the BVHs of num_scenes scenes with one launch per LBVH stage across all of them
 * (leaf boxes and per-scene bounds, Morton codes, one stable sort of every code plus one
 * stable pass on the scene index, the radix trees, the refits); treelet rounds and the
 * traversal layout then run per scene.  out[k] is identical to cav_bvh_build of scene k
 * alone.  positions[k], indices[k], mesh_ids[k] (mesh_ids may be NULL) are DEVICE arrays;
 * num_vertices, num_triangles: host arrays (vertex indices are checked against num_vertices
 * as in cav_bvh_build); scene_bounds: NULL (computed) or num_scenes x 6 host floats.  At
 * most 65,536 scenes and 2^32 triangles in total. */
cav_status cav_bvh_build_batch(cav_ctx* ctx, int num_scenes, const float* const* positions,
                               const int64_t* num_vertices, const int32_t* const* indices,
                               const int32_t* const* mesh_ids, const int64_t* num_triangles,
                               const float* scene_bounds, int rounds, void* stream, cav_bvh** out);

/* Device-side event timing of the last build's stages (ms): leaf boxes + Morton,
 * sort, radix tree, refit, treelet rounds, layout.  Valid after the stream is synced. */
cav_status cav_bvh_stage_times(cav_ctx* ctx, const cav_bvh* bvh, float* ms6);

#ifdef __cplusplus
}
#endif

#endif /* CAVALRY_B200_H */
