// Internal declarations shared by the cavalry_b200 CUDA translation units.
//
// All translation units are compiled with -use_fast_math (the reference's numerics
// flags, CMakeLists.txt:5), so divisions, reciprocals and multiply-adds behave as in
// the reference's kernels; floating-point expressions that feed bit-exact outputs are
// written in the same operand order as the reference.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>

#include "../../include/cavalry.h"

namespace cav {

// ----------------------------------------------------------------- vectors
struct f3 {
    float x, y, z;
};
__host__ __device__ inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ inline f3 operator/(f3 a, f3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
__host__ __device__ inline f3 vmin3(f3 a, f3 b) { return mk(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__host__ __device__ inline f3 vmax3(f3 a, f3 b) { return mk(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
// Same operand order as the reference's cross/dot (helper math of Core/Triangle.h:7-57).
__host__ __device__ inline f3 cross3(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// AABB::computeSurfaceArea, Core/BoundingBox.h:77-80 (same expression).
__device__ inline float surface_area(f3 lo, f3 hi) {
    f3 e = hi - lo;
    return 2.f * (e.x * e.y + e.y * e.z + e.x * e.z);
}
// BVH/SAH.h:4-22: FP64 literals, float results.
__device__ inline float leaf_cost(float area, int n) { return area * 1.0 * n; }
__device__ inline float internal_cost(float area, float l, float r) { return area * 1.2 + l + r; }
__device__ inline float internal_cost(float area, float c) { return area * 1.2 + c; }

// Build error bits, or-ed into the context's first error word by a build and mapped to a
// cav_status by cav_sync_check.  Every bit but kErrBadIndex means the tree's structure is not
// to be trusted (the sort's permutation, the radix tree or the refit broke): the build's
// later kernels then check every index they take from it, and its last kernel replaces the
// traversal root with one that no ray hits, so a failed tree is still safe to trace.
constexpr int kErrLookback = 1;     // sort look-back wait gave up
constexpr int kErrSortScatter = 2;  // a sort scatter position broke an invariant
constexpr int kErrRadixSplit = 4;   // a radix-tree split fell outside its range
constexpr int kErrBadIndex = 8;     // a triangle's vertex index is outside [0, num_vertices)
constexpr int kErrRefitLink = 16;   // the refit met a parent, child or leaf index outside the tree
constexpr int kErrStructural = kErrLookback | kErrSortScatter | kErrRadixSplit | kErrRefitLink;

// ------------------------------------------------------------ node records
// Build/restructure node (64 bytes).  Internal nodes at [0, N-2] after the build,
// leaf j (sorted position) at N-1+j; treelet rounds permute roles among ids.
struct __align__(16) BNode {
    float lo_x, lo_y, lo_z, hi_x;  // 16
    float hi_y, hi_z;              // 24
    int32_t left, right;           // 32
    int32_t parent, prim;          // 40 (prim: triangle id of a leaf, -1 internal)
    float area, cost;              // 48
    int32_t is_leaf, pad0;         // 56
    int32_t pad1, pad2;            // 64
};
static_assert(sizeof(BNode) == 64, "BNode must be 64 bytes");

// Traversal node (64 bytes): both children's boxes, fetched with four 16-byte loads.
// child ref >= 0: internal node index; < 0: ~(triangle slot).
struct __align__(64) TNode {
    float4 a;  // L.lo.x L.lo.y L.lo.z L.hi.x
    float4 b;  // L.hi.y L.hi.z R.lo.x R.lo.y
    float4 c;  // R.lo.z R.hi.x R.hi.y R.hi.z
    int4 d;    // left ref, right ref, 0, 0
};
static_assert(sizeof(TNode) == 64, "TNode must be 64 bytes");

// Compressed 8-wide traversal node (80 bytes) of the fast mode, after Ylitie, Karras and
// Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs" (HPG
// 2017).  Child boxes are 8-bit offsets on a per-node grid: plane = p + q * 2^(e - 127) per
// axis, rounded outward when quantised.  Internal children are stored contiguously from
// child_base in slot order (imask bit s = slot s holds an internal child); triangle children
// contiguously from tri_base.  meta[s]: 0 = empty slot; 0x20 | (24 + s) = internal child;
// 0x20 | k = triangle tri_base + k.  A child's slot is chosen so that the slot number's bits
// give the side of the node's centre it lies on (bit 2: +x, bit 1: +y, bit 0: +z), which lets
// a ray visit children near-first by its direction octant alone.
struct __align__(16) CNode {
    float px, py, pz;
    uint32_t e_imask;  // biased exponents x | y << 8 | z << 16, imask << 24
    uint32_t child_base, tri_base;
    uint32_t meta[2];  // slots 0-3, 4-7 (one byte each)
    uint32_t qlo_x[2], qlo_y[2];
    uint32_t qlo_z[2], qhi_x[2];
    uint32_t qhi_y[2], qhi_z[2];
};
static_assert(sizeof(CNode) == 80, "CNode must be 80 bytes");

// Triangle record (48 bytes) in sorted (Morton) order: v0, e1 = v1-v0, e2 = v2-v0
// (the same subtractions as Core/Triangle.h:180-183), triangle id and mesh id.
struct __align__(16) TriRec {
    float4 v0;  // v0.xyz, id (int bits)
    float4 e1;  // e1.xyz, mesh id (int bits)
    float4 e2;  // e2.xyz, 0
};
static_assert(sizeof(TriRec) == 48, "TriRec must be 48 bytes");

}  // namespace cav

// ------------------------------------------------------------ host objects
struct cav_ctx {
    int device = 0;
    int num_sms = 148;
    std::string last_error;
    // traversal launch configuration (0 = defaults)
    int trace_block = 0;
    int trace_blocks_per_sm = 0;
    int trace_batch = 0;
    int trace_stack = 0;  // 64 selects the short traversal stack for trees known to be shallow
    int trace_smem_stack = 0;  // > 0: the first stack entries of the exact kernels in shared memory
    // bounded device-side waits (cav_ctx_set_limits)
    uint32_t max_trace_steps = 1u << 22;     // node + triangle visits allowed one ray
    uint64_t sort_wait_ns = 2000000000ull;  // a sort tile's look-back wait, and a tcgen05 completion wait
    // failure injection for tests (cav_ctx_inject); lanes of a server read them concurrently
    std::atomic<int> inject_sort_stall{0};
    std::atomic<int> inject_alloc_fail{0};  // k > 0: the k-th next device allocation fails
    std::atomic<int> inject_mlp_stall{0};   // the tcgen05 MLP forward skips each group's first commit
    // launch configuration of the fast (compressed 8-wide) mode (0 = defaults)
    int wide_block = 0;
    int wide_batch = 0;
    int wide_smem_stack = 0;  // > 0: the fast mode's first stack entries in shared memory
    // persistent work counters (device), one per concurrent trace kind
    unsigned long long* d_counters = nullptr;
    int* d_error = nullptr;
    // host-path staging
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    void* dev_stage = nullptr;
    size_t dev_stage_bytes = 0;
    cudaStream_t hstream[2] = {nullptr, nullptr};
    cudaEvent_t hevent[2] = {nullptr, nullptr};
    // Halton tables on the device, uploaded by the first scene and shared by all
    std::mutex halton_mu;
    uint32_t* d_halton_primes = nullptr;
    uint32_t* d_halton_start = nullptr;
    uint16_t* d_halton_perms = nullptr;
};

namespace cav {
// A device allocation shared by the trees of one batched build; the last tree released frees it.
struct SharedArena {
    void* p = nullptr;
    std::atomic<int> refs{0};
};
}  // namespace cav

struct cav_bvh {
    int64_t n = 0;  // triangles
    mutable int32_t depth = -1;  // tree depth once measured (cav_bvh_depth), else -1
    int device = 0;
    // build products
    cav::BNode* nodes = nullptr;       // 2N-1 restructure records (reference order)
    uint64_t* codes_unsorted = nullptr;  // N
    uint64_t* codes_sorted = nullptr;    // N
    int32_t* perm = nullptr;             // N: sorted position -> triangle id
    // traversal layout
    cav::TNode* tnodes = nullptr;  // N-1
    // compressed 8-wide view for CAV_TRACE_FAST, built on first use (wide.cu)
    mutable cav::CNode* cnodes = nullptr;
    mutable cav::TriRec* ctris = nullptr;  // triangles in wide-leaf order
    mutable void* wide_arena = nullptr;
    cav::TriRec* tris = nullptr;   // N
    float root_box[6];             // copied to the host at build time? no: device copy
    float* d_root_box = nullptr;   // 6 floats on device
    int32_t* d_depth = nullptr;    // scratch for cav_bvh_depth
    float stage_ms[6] = {0, 0, 0, 0, 0, 0};
    cudaEvent_t ev[7] = {};
    bool timed = false;
    void* arena = nullptr;  // one allocation holding the arrays above (null when shared)
    cav::SharedArena* shared = nullptr;  // the batch's arena the arrays live in, or null
};

namespace cav {

cav_status set_error(cav_ctx* ctx, cav_status s, const std::string& msg);
cav_status cuda_error(cav_ctx* ctx, cudaError_t e, const char* what);
// A device allocation made for a context: stream-ordered on `s` when `async`, else plain.
// Fails with cudaErrorMemoryAllocation while the context's injected allocation failures last
// (cav_ctx_inject), so the error paths of every caller can be tested without exhausting HBM.
cudaError_t dev_alloc(cav_ctx* ctx, void** p, size_t bytes, cudaStream_t s, bool async);

// build.cu
// Releases a tree (cav_bvh_free); async: stream-ordered frees on `s`, for callers (the
// server) that must not wait for the device.
void bvh_release(cav_bvh* bvh, cudaStream_t s, bool async);
size_t bvh_arena_bytes(int64_t n);
cav_status build_bvh(cav_ctx* ctx, const float* positions, int64_t nv, const int32_t* indices,
                     const int32_t* mesh_ids, int64_t n, const float* bounds, int rounds, cudaStream_t s,
                     cav_bvh** out);
// Stable LSD radix sort of (key, value) pairs by the low 8 * passes bits of the keys (passes
// even, so the result ends in keys / vals), with the build's kernels: keys_tmp / vals_tmp hold
// n entries, hist 8 x 256 words, status sort_status_words(n, passes) words, counters `passes`
// words; all are cleared here.  A look-back wait that runs out sets kErrLookback in *err.
size_t sort_status_words(int64_t n, int passes);
cav_status sort_pairs(cav_ctx* ctx, uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                      int passes, uint32_t* hist, uint32_t* status, uint32_t* counters, int* err, cudaStream_t s);
// treelet.cu
// counters: device words of the caller's scratch ([0]: leaf-list positions, [1]: the walkers' claims)
cav_status treelet_rounds(cav_ctx* ctx, BNode* nodes, int64_t n, int rounds, int32_t* leaf_list, uint32_t* visited,
                          uint32_t* counters, cudaStream_t s);
struct TreeletSeg {  // one tree of a batched treelet pass
    BNode* nodes;
    int64_t n;  // leaves (triangles)
};
cav_status treelet_rounds_batch(cav_ctx* ctx, const TreeletSeg* segs, const TreeletSeg* segs_host,
                                const int64_t* leaf_off, const int64_t* leaf_off_host, int K, int rounds,
                                int32_t* leaf_list, uint32_t* counters, uint32_t* visited, cudaStream_t s);
// trace.cu
// A traversal segment: one job's rays against one tree, with its own outputs.  `begin` is
// the segment's first index in the launch's global ray numbering.
struct TraceSeg {
    const TNode* nodes;
    const TriRec* tris;
    const float* root_box;
    const cav_ray* rays;
    int32_t* prim;     // closest hit
    float* t;
    float* uv;
    const float* limit;  // any hit
    const int32_t* excl;
    uint8_t* occ;
    int64_t begin;
    const uint32_t* n_dev;  // single-tree launches: ray count read from device memory (or null)
    const CNode* cnodes;    // the tree's compressed 8-wide view (fast-mode launches; ensure_wide)
    const TriRec* ctris;
};
cav_status trace_closest_segments(cav_ctx* ctx, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags,
                                  cudaStream_t s, unsigned long long* counter);
cav_status trace_any_segments(cav_ctx* ctx, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags, cudaStream_t s,
                              unsigned long long* counter);
int trace_max_segments();
// Single-tree traversal whose ray count is read from device memory at launch (n_dev),
// n_max bounding it; for launch chains without host round trips (CUDA graphs).
cav_status trace_closest_dev(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const uint32_t* n_dev,
                             int32_t* prim, float* t, float* uv, cudaStream_t s, unsigned long long* counter);
cav_status trace_any_dev(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                         const int32_t* excl, const uint32_t* n_dev, uint8_t* occ, cudaStream_t s,
                         unsigned long long* counter);

// Compressed 8-wide fast mode (wide.cu): the layout is built on the stream at first use.
cav_status ensure_wide(cav_ctx* ctx, const cav_bvh* bvh, cudaStream_t s);
// stats (2 counters: node visits, triangle tests), when given, selects the instrumented variant
cav_status trace_wide_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n,
                              const uint32_t* n_dev, int32_t* prim, float* t, float* uv, cudaStream_t s,
                              unsigned long long* counter, unsigned long long* stats = nullptr);
cav_status trace_wide_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                          const int32_t* excl, int64_t n, const uint32_t* n_dev, uint8_t* occ, cudaStream_t s,
                          unsigned long long* counter, unsigned long long* stats = nullptr);
void free_wide(cav_bvh* bvh, cudaStream_t s, bool async);
cav_status trace_wide_segments(cav_ctx* ctx, bool any_hit, const TraceSeg* segs, int nseg, int64_t n, cudaStream_t s,
                               unsigned long long* counter);

// render.cu: scenes that a job brings (the server uploads, builds and releases them on its
// stream), and the graph-replayed render
}  // namespace cav
namespace cavpbrt {
struct Scene;
}
namespace cav {
cav_status scene_upload(cav_ctx* ctx, cavpbrt::Scene&& desc, cudaStream_t s, bool async, cav_scene** out);
void scene_release(cav_scene* sc, cudaStream_t s, bool async);
size_t scene_device_bytes(const cavpbrt::Scene& desc);
// The scene's device geometry (the inputs of its BVH build) and the tree it traverses.
void scene_geometry(const cav_scene* sc, const float** pos, int64_t* nv, const int32_t** idx, const int32_t** mesh,
                    int64_t* nt);
void scene_set_bvh(cav_scene* sc, cav_bvh* bvh, int rounds);
int scene_spp(const cav_scene* sc);
// counters: two device words for the traversals' work counters (null: the context's)
cav_status render_path_graph(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                             cudaStream_t s, unsigned long long* counters = nullptr);

// Many scenes' BVHs, one launch per LBVH stage across all of them (build.cu)
cav_status build_bvh_batch(cav_ctx* ctx, int K, const float* const* positions, const int64_t* num_vertices,
                           const int32_t* const* indices, const int32_t* const* mesh_ids, const int64_t* num_triangles,
                           const float* bounds, int rounds, cudaStream_t s, cav_bvh** out);

// MLP forward pass for the guided integrator (mlp.cu): in n x 5 -> out n x 32
cav_status mlp_forward(cav_mlp* m, const float* in, int64_t n, float* out, cudaStream_t s);

// Resumable path-integrator render (render.cu), advanced bounce by bounce by the server.
struct PathJob;
size_t path_job_bytes(const cav_scene* sc, const cav_render_opts* opts);
// Path state + film of a W x H x spp render in chunks of max_paths (<= 0: 4M) paths.
size_t render_state_bytes(int W, int H, int spp, int64_t max_paths);
cav_status path_job_create(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, int64_t slice, cudaStream_t s,
                           PathJob** out);
void path_job_set_slice(PathJob* J, int64_t slice);
int64_t path_job_capacity(const PathJob* J);
int64_t path_job_extend(PathJob* J, TraceSeg* seg);
cav_status path_job_shade(PathJob* J, cudaStream_t s);
int64_t path_job_shadow(PathJob* J, TraceSeg* seg);
cav_status path_job_advance(PathJob* J, cudaStream_t s, bool* finished);
void path_job_film(PathJob* J, float** sum, float** wsum, int64_t* pixels);
void path_job_destroy(PathJob* J, cudaStream_t s);
cav_status trace_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int32_t* prim, float* t,
                         float* uv, uint32_t flags, cudaStream_t s, unsigned long long* counter);
cav_status trace_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                     const int32_t* excl, int64_t n, uint8_t* occ, uint32_t flags, cudaStream_t s,
                     unsigned long long* counter);
cav_status trace_stats(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                       const float* limit, const int32_t* excl, uint32_t flags, cudaStream_t s, uint64_t* host2);

#define CAV_CUDA(ctx, call)                                              \
    do {                                                                 \
        cudaError_t e__ = (call);                                        \
        if (e__ != cudaSuccess) return ::cav::cuda_error(ctx, e__, #call); \
    } while (0)

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace cav
