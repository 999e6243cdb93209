// C ABI of cavalry_b200 (declared in include/cavalry.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "cav_internal.cuh"
#include "trace_common.cuh"

namespace cav {

cav_status set_error(cav_ctx* ctx, cav_status s, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return s;
}

cudaError_t dev_alloc(cav_ctx* ctx, void** p, size_t bytes, cudaStream_t s, bool async) {
    int left = ctx->inject_alloc_fail.load();
    while (left > 0) {  // count down to the injected failure
        if (ctx->inject_alloc_fail.compare_exchange_weak(left, left - 1)) {
            if (left == 1) return cudaErrorMemoryAllocation;
            break;
        }
    }
    return async ? cudaMallocAsync(p, bytes, s) : cudaMalloc(p, bytes);
}

cav_status cuda_error(cav_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, m);
    return set_error(ctx, CAV_ERR_CUDA, m);
}

}  // namespace cav

using namespace cav;

namespace {

constexpr int kCounterWords = 64;
constexpr int kErrorWords = 16;

cav_status use_device(cav_ctx* ctx) {
    if (!ctx) return CAV_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
    return CAV_OK;
}

bool is_pinned_host(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

int cav_version(void) { return 10000; }

const char* cav_status_string(cav_status s) {
    switch (s) {
        case CAV_OK: return "ok";
        case CAV_ERR_INVALID_ARGUMENT: return "invalid argument";
        case CAV_ERR_CUDA: return "CUDA error";
        case CAV_ERR_OUT_OF_MEMORY: return "out of device memory";
        case CAV_ERR_TIMEOUT: return "device-side wait timed out";
        case CAV_ERR_STACK_OVERFLOW: return "traversal stack overflow";
        case CAV_ERR_NOT_READY: return "not ready";
        case CAV_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

cav_status cav_ctx_create(int device, cav_ctx** out) {
    if (!out) return CAV_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    cav_ctx* ctx = new (std::nothrow) cav_ctx();
    if (!ctx) return CAV_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return CAV_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    // Renders allocate their path state stream-ordered (cudaMallocAsync from the device's
    // default pool); keep freed pool memory mapped instead of releasing it at every
    // synchronisation, so repeated renders do not map gigabytes again each call.
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess && pool) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    if (cudaMalloc(&ctx->d_counters, sizeof(unsigned long long) * kCounterWords) != cudaSuccess ||
        cudaMalloc(&ctx->d_error, sizeof(int) * kErrorWords) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(ctx->d_counters);
        delete ctx;
        return CAV_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(ctx->d_counters, 0, sizeof(unsigned long long) * kCounterWords);
    cudaMemset(ctx->d_error, 0, sizeof(int) * kErrorWords);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    *out = ctx;
    return CAV_OK;
}

cav_status cav_ctx_destroy(cav_ctx* ctx) {
    if (!ctx) return CAV_OK;
    cudaSetDevice(ctx->device);
    for (int k = 0; k < 2; ++k) {
        if (ctx->hstream[k]) cudaStreamDestroy(ctx->hstream[k]);
        if (ctx->hevent[k]) cudaEventDestroy(ctx->hevent[k]);
    }
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->dev_stage) cudaFree(ctx->dev_stage);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_halton_primes);
    cudaFree(ctx->d_halton_start);
    cudaFree(ctx->d_halton_perms);
    delete ctx;
    return CAV_OK;
}

const char* cav_last_error(const cav_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

cav_status cav_set_trace_config(cav_ctx* ctx, int block_threads, int blocks_per_sm, int batch) {
    if (!ctx) return CAV_ERR_INVALID_ARGUMENT;
    if (block_threads < 0 || block_threads > 1024 || (block_threads % 32) != 0 || blocks_per_sm < 0 ||
        blocks_per_sm > 64 || batch < 0 || batch > 32)
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_set_trace_config: out of range");
    ctx->trace_block = block_threads;
    ctx->trace_blocks_per_sm = blocks_per_sm;
    ctx->trace_batch = batch;
    return CAV_OK;
}

cav_status cav_set_trace_stack(cav_ctx* ctx, uint32_t flags, int stack, int smem_stack) {
    if (!ctx) return CAV_ERR_INVALID_ARGUMENT;
    if (flags & CAV_TRACE_FAST) {
        if (flags != CAV_TRACE_FAST || stack != 0 || (smem_stack != 0 && smem_stack != kWideSmemStack))
            return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_set_trace_stack: fast mode takes stack 0, smem_stack 0/8");
        ctx->wide_smem_stack = smem_stack;
        return CAV_OK;
    }
    if (flags != CAV_TRACE_EXACT || (stack != 0 && stack != 64 && stack != 128) ||
        (smem_stack != 0 && smem_stack != 16))
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_set_trace_stack: stack 0/64/128, smem_stack 0/16");
    ctx->trace_stack = stack;
    ctx->trace_smem_stack = smem_stack;
    return CAV_OK;
}

cav_status cav_bvh_build_batch(cav_ctx* ctx, int num_scenes, const float* const* positions,
                               const int64_t* num_vertices, const int32_t* const* indices,
                               const int32_t* const* mesh_ids, const int64_t* num_triangles,
                               const float* scene_bounds, int rounds, void* stream, cav_bvh** out) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    return build_bvh_batch(ctx, num_scenes, positions, num_vertices, indices, mesh_ids, num_triangles, scene_bounds,
                           rounds, (cudaStream_t)stream, out);
}

cav_status cav_bvh_build(cav_ctx* ctx, const float* positions, int64_t num_vertices, const int32_t* indices,
                         const int32_t* mesh_ids, int64_t num_triangles, const float* scene_bounds, int rounds,
                         void* stream, cav_bvh** out) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (out) *out = nullptr;
    return build_bvh(ctx, positions, num_vertices, indices, mesh_ids, num_triangles, scene_bounds, rounds,
                     (cudaStream_t)stream, out);
}

cav_status cav_bvh_free(cav_bvh* bvh) {
    if (!bvh) return CAV_OK;
    cudaSetDevice(bvh->device);
    cav::bvh_release(bvh, nullptr, false);
    return CAV_OK;
}

int64_t cav_bvh_num_triangles(const cav_bvh* bvh) { return bvh ? bvh->n : 0; }

int cav_bvh_has_fast_layout(const cav_bvh* bvh) { return bvh && bvh->cnodes ? 1 : 0; }

cav_status cav_bvh_stage_times(cav_ctx* ctx, const cav_bvh* bvh, float* ms6) {
    if (!ctx || !bvh || !ms6) return CAV_ERR_INVALID_ARGUMENT;
    if (!bvh->timed) return set_error(ctx, CAV_ERR_NOT_READY, "no timing recorded");
    for (int k = 0; k < 6; ++k) {
        cudaError_t e = cudaEventElapsedTime(&ms6[k], bvh->ev[k], bvh->ev[k + 1]);
        if (e != cudaSuccess) return cuda_error(ctx, e, "cudaEventElapsedTime");
    }
    return CAV_OK;
}

cav_status cav_bvh_export_nodes(cav_ctx* ctx, const cav_bvh* bvh, void* stream, cav_ref_node* host_out) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (!bvh || !host_out) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_export_nodes: null");
    const int64_t count = 2 * bvh->n - 1;
    std::vector<BNode> h((size_t)count);
    CAV_CUDA(ctx, cudaMemcpyAsync(h.data(), bvh->nodes, sizeof(BNode) * count, cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream));
    CAV_CUDA(ctx, cudaStreamSynchronize((cudaStream_t)stream));
    for (int64_t i = 0; i < count; ++i) {
        const BNode& b = h[(size_t)i];
        cav_ref_node& o = host_out[i];
        o.bmin[0] = b.lo_x; o.bmin[1] = b.lo_y; o.bmin[2] = b.lo_z;
        o.bmax[0] = b.hi_x; o.bmax[1] = b.hi_y; o.bmax[2] = b.hi_z;
        o.prim_begin = b.is_leaf ? b.prim : -1;
        o.prim_end = b.is_leaf ? b.prim : -1;
        o.left = b.left;
        o.right = b.right;
        o.is_leaf = b.is_leaf ? 1 : 0;
    }
    return CAV_OK;
}

cav_status cav_bvh_export_stages(cav_ctx* ctx, const cav_bvh* bvh, void* stream, uint64_t* morton_unsorted,
                                 uint64_t* morton_sorted, int32_t* sorted_prims) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (!bvh) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_export_stages: null");
    cudaStream_t s = (cudaStream_t)stream;
    if (morton_unsorted)
        CAV_CUDA(ctx, cudaMemcpyAsync(morton_unsorted, bvh->codes_unsorted, 8 * bvh->n, cudaMemcpyDeviceToHost, s));
    if (morton_sorted)
        CAV_CUDA(ctx, cudaMemcpyAsync(morton_sorted, bvh->codes_sorted, 8 * bvh->n, cudaMemcpyDeviceToHost, s));
    if (sorted_prims) CAV_CUDA(ctx, cudaMemcpyAsync(sorted_prims, bvh->perm, 4 * bvh->n, cudaMemcpyDeviceToHost, s));
    CAV_CUDA(ctx, cudaStreamSynchronize(s));
    return CAV_OK;
}

cav_status cav_bvh_depth(cav_ctx* ctx, const cav_bvh* bvh, void* stream, int32_t* depth) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (!bvh || !depth) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_depth: null");
    const int64_t count = 2 * bvh->n - 1;
    std::vector<BNode> h((size_t)count);
    CAV_CUDA(ctx, cudaMemcpyAsync(h.data(), bvh->nodes, sizeof(BNode) * count, cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream));
    CAV_CUDA(ctx, cudaStreamSynchronize((cudaStream_t)stream));
    std::vector<std::pair<int32_t, int32_t>> stk;
    stk.push_back({0, 0});
    int32_t best = 0;
    int64_t guard = 0;
    while (!stk.empty()) {
        auto [x, d] = stk.back();
        stk.pop_back();
        if (x < 0 || x >= count || ++guard > 2 * count + 2)
            return set_error(ctx, CAV_ERR_CUDA, "cav_bvh_depth: malformed tree");
        best = std::max(best, d);
        if (!h[(size_t)x].is_leaf) {
            stk.push_back({h[(size_t)x].left, d + 1});
            stk.push_back({h[(size_t)x].right, d + 1});
        }
    }
    *depth = best;
    bvh->depth = best;
    return CAV_OK;
}

// Synchronises `stream` and reports device-side error flags raised since the last check
// (sort look-back timeout, treelet inconsistency, traversal stack overflow), clearing them.
cav_status cav_sync_check(cav_ctx* ctx, void* stream) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    int flags[kErrorWords];
    CAV_CUDA(ctx, cudaStreamSynchronize((cudaStream_t)stream));
    CAV_CUDA(ctx, cudaMemcpy(flags, ctx->d_error, sizeof(flags), cudaMemcpyDeviceToHost));
    CAV_CUDA(ctx, cudaMemset(ctx->d_error, 0, sizeof(flags)));
    if (flags[0] & kErrLookback)
        return set_error(ctx, CAV_ERR_TIMEOUT, "radix sort look-back wait gave up (the tree reports no hits)");
    if (flags[0] & kErrBadIndex)
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_build: a vertex index is outside [0, num_vertices)");
    if (flags[0])
        return set_error(ctx, CAV_ERR_CUDA, "BVH build: a sort, radix-tree or refit invariant broke (the tree reports "
                                            "no hits)");
    if (flags[1]) return set_error(ctx, CAV_ERR_CUDA, "treelet reconstruction found an inconsistent partition");
    if ((flags[2] | flags[3]) & kFlagStackOverflow)
        return set_error(ctx, CAV_ERR_STACK_OVERFLOW, "traversal stack overflow");
    if ((flags[2] | flags[3]) & kFlagStepLimit)
        return set_error(ctx, CAV_ERR_TIMEOUT, "traversal step limit reached (rays stopped)");
    if (flags[4]) return set_error(ctx, CAV_ERR_TIMEOUT, "MLP forward: a tensor-core completion wait gave up");
    if (flags[5] & kErrLookback)
        return set_error(ctx, CAV_ERR_TIMEOUT, "ray reordering: the sort's look-back wait gave up (results not meaningful)");
    if (flags[5]) return set_error(ctx, CAV_ERR_CUDA, "ray reordering: a sort invariant broke (results not meaningful)");
    return CAV_OK;
}

cav_status cav_ctx_set_limits(cav_ctx* ctx, double sort_wait_s, int64_t max_trace_steps) {
    if (!ctx) return CAV_ERR_INVALID_ARGUMENT;
    if (sort_wait_s > 60.0 || max_trace_steps > (int64_t)UINT32_MAX)
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_ctx_set_limits: out of range");
    ctx->sort_wait_ns = sort_wait_s > 0 ? (uint64_t)(sort_wait_s * 1e9) : 2000000000ull;
    ctx->max_trace_steps = max_trace_steps > 0 ? (uint32_t)max_trace_steps : kMaxSteps;
    return CAV_OK;
}

cav_status cav_ctx_inject(cav_ctx* ctx, int what, int count) {
    if (!ctx || count < 0) return CAV_ERR_INVALID_ARGUMENT;
    switch (what) {
        case CAV_INJECT_NONE:
            ctx->inject_sort_stall = 0;
            ctx->inject_alloc_fail = 0;
            ctx->inject_mlp_stall = 0;
            return CAV_OK;
        case CAV_INJECT_SORT_STALL:
            ctx->inject_sort_stall = count > 0 ? 1 : 0;
            return CAV_OK;
        case CAV_INJECT_ALLOC_FAIL:
            ctx->inject_alloc_fail = count;
            return CAV_OK;
        case CAV_INJECT_MLP_STALL:
            ctx->inject_mlp_stall = count > 0 ? 1 : 0;
            return CAV_OK;
        default:
            return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_ctx_inject: unknown failure");
    }
}

cav_status cav_trace_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int32_t* prim_id,
                             float* t, float* uv, uint32_t flags, void* stream) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    return trace_closest(ctx, bvh, rays, n, prim_id, t, uv, flags, (cudaStream_t)stream, ctx->d_counters + 0);
}

cav_status cav_trace_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                         const int32_t* excl_mesh, int64_t n, uint8_t* occluded, uint32_t flags, void* stream) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    return trace_any(ctx, bvh, rays, limit, excl_mesh, n, occluded, flags, (cudaStream_t)stream, ctx->d_counters + 1);
}

cav_status cav_trace_stats(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                           const float* limit, const int32_t* excl_mesh, uint32_t flags, void* stream,
                           uint64_t* host_counts) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    return trace_stats(ctx, bvh, rays, n, any_hit, limit, excl_mesh, flags, (cudaStream_t)stream, host_counts);
}

}  // extern "C"

// ------------------------------------------------------------ host-buffer path
namespace {

// Rays per pipelined chunk.  Every traversal launch ends in a tail while its last, longest
// rays finish (about 4.7 ms on the 1M-triangle soup), so chunks are large: 4M rays of the
// soup take 68.4 ms through the host path in one chunk against 76.9 ms in four chunks of 1M
// (64.9 ms of traversal alone).
constexpr int64_t kChunkRays = (int64_t)1 << 22;
// per-ray staging bytes: ray 32 + limit 4 + excl 8 in; prim 4 + t 4 + uv 8 (or occ 1) out
constexpr size_t kInBytes = 32 + 4 + 8;
constexpr size_t kOutBytes = 16;
constexpr size_t kSlotBytes = (kInBytes + kOutBytes) * kChunkRays + 4096;

// The host-buffer entry points run on the context's own streams; they first wait for the
// BVH's build (recorded on the caller's build stream) to complete.
cav_status order_after_build(cav_ctx* ctx, const cav_bvh* bvh) {
    if (!bvh->timed) return CAV_OK;
    for (int k = 0; k < 2; ++k) CAV_CUDA(ctx, cudaStreamWaitEvent(ctx->hstream[k], bvh->ev[6], 0));
    return CAV_OK;
}

// Device staging (two slots) always; pinned host staging only once a call passes a pageable
// host buffer (pinned caller buffers are copied directly).
cav_status ensure_host_path(cav_ctx* ctx, bool need_pinned) {
    if (!ctx->hstream[0]) {
        for (int k = 0; k < 2; ++k) {
            CAV_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->hstream[k], cudaStreamNonBlocking));
            CAV_CUDA(ctx, cudaEventCreateWithFlags(&ctx->hevent[k], cudaEventDisableTiming));
        }
    }
    if (!ctx->dev_stage) {
        CAV_CUDA(ctx, cudaMalloc(&ctx->dev_stage, 2 * kSlotBytes));
        ctx->dev_stage_bytes = 2 * kSlotBytes;
    }
    if (need_pinned && !ctx->pinned) {
        CAV_CUDA(ctx, cudaMallocHost(&ctx->pinned, 2 * kSlotBytes));
        ctx->pinned_bytes = 2 * kSlotBytes;
    }
    return CAV_OK;
}

struct Slot {
    unsigned char* d;  // device slot base
    unsigned char* h;  // pinned slot base
    cav_ray* d_rays;
    float* d_lim;
    int32_t* d_excl;
    unsigned char* d_out;
    cav_ray* h_rays;
    float* h_lim;
    int32_t* h_excl;
    unsigned char* h_out;
};

Slot slot_of(cav_ctx* ctx, int k) {
    Slot s;
    s.d = (unsigned char*)ctx->dev_stage + k * kSlotBytes;
    size_t off_lim = 32 * kChunkRays, off_excl = off_lim + 4 * kChunkRays, off_out = off_excl + 8 * kChunkRays;
    s.d_rays = (cav_ray*)s.d;
    s.d_lim = (float*)(s.d + off_lim);
    s.d_excl = (int32_t*)(s.d + off_excl);
    s.d_out = s.d + off_out;
    // pinned slots exist only once a pageable buffer has been passed (ensure_host_path)
    s.h = ctx->pinned ? (unsigned char*)ctx->pinned + k * kSlotBytes : nullptr;
    s.h_rays = s.h ? (cav_ray*)s.h : nullptr;
    s.h_lim = s.h ? (float*)(s.h + off_lim) : nullptr;
    s.h_excl = s.h ? (int32_t*)(s.h + off_excl) : nullptr;
    s.h_out = s.h ? s.h + off_out : nullptr;
    return s;
}

// Pipelined chunk loop: H2D of chunk c+1 overlaps traversal of chunk c and D2H of c-1
// on two streams.  Inputs already in pinned memory are copied directly; pageable
// inputs and outputs go through the context's pinned slots.
template <typename Launch, typename Finish>
cav_status host_pipeline(cav_ctx* ctx, int64_t n, Launch launch, Finish finish) {
    const int64_t chunks = (n + kChunkRays - 1) / kChunkRays;
    int64_t pending[2] = {-1, -1};
    for (int64_t c = 0; c < chunks; ++c) {
        const int k = (int)(c & 1);
        if (pending[k] >= 0) {
            CAV_CUDA(ctx, cudaEventSynchronize(ctx->hevent[k]));
            cav_status st = finish(slot_of(ctx, k), pending[k]);
            if (st != CAV_OK) return st;
            pending[k] = -1;
        }
        cav_status st = launch(slot_of(ctx, k), c, ctx->hstream[k], ctx->d_counters + 2 + k);
        if (st != CAV_OK) return st;
        CAV_CUDA(ctx, cudaEventRecord(ctx->hevent[k], ctx->hstream[k]));
        pending[k] = c;
    }
    for (int k = 0; k < 2; ++k) {
        if (pending[k] < 0) continue;
        CAV_CUDA(ctx, cudaEventSynchronize(ctx->hevent[k]));
        cav_status st = finish(slot_of(ctx, k), pending[k]);
        if (st != CAV_OK) return st;
    }
    return CAV_OK;
}

}  // namespace

extern "C" {

cav_status cav_trace_closest_host(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int32_t* prim_id,
                                  float* t, float* uv, uint32_t flags) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (!bvh || !rays || !prim_id || n < 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_trace_closest_host");
    if (n == 0) return CAV_OK;
    const bool in_pinned = is_pinned_host(rays);
    const bool out_pinned = is_pinned_host(prim_id) && (!t || is_pinned_host(t)) && (!uv || is_pinned_host(uv));
    st = ensure_host_path(ctx, !(in_pinned && out_pinned));
    if (st != CAV_OK) return st;
    st = order_after_build(ctx, bvh);
    if (st != CAV_OK) return st;
    auto launch = [&](Slot s, int64_t c, cudaStream_t str, unsigned long long* counter) -> cav_status {
        int64_t b = c * kChunkRays, m = std::min(kChunkRays, n - b);
        if (in_pinned) {
            CAV_CUDA(ctx, cudaMemcpyAsync(s.d_rays, rays + b, 32 * m, cudaMemcpyHostToDevice, str));
        } else {
            memcpy(s.h_rays, rays + b, 32 * m);
            CAV_CUDA(ctx, cudaMemcpyAsync(s.d_rays, s.h_rays, 32 * m, cudaMemcpyHostToDevice, str));
        }
        int32_t* dp = (int32_t*)s.d_out;
        float* dt = (float*)(s.d_out + 4 * kChunkRays);
        float* duv = (float*)(s.d_out + 8 * kChunkRays);
        cav_status r = trace_closest(ctx, bvh, s.d_rays, m, dp, t ? dt : nullptr, uv ? duv : nullptr, flags, str,
                                     counter);
        if (r != CAV_OK) return r;
        if (out_pinned) {
            CAV_CUDA(ctx, cudaMemcpyAsync(prim_id + b, dp, 4 * m, cudaMemcpyDeviceToHost, str));
            if (t) CAV_CUDA(ctx, cudaMemcpyAsync(t + b, dt, 4 * m, cudaMemcpyDeviceToHost, str));
            if (uv) CAV_CUDA(ctx, cudaMemcpyAsync(uv + 2 * b, duv, 8 * m, cudaMemcpyDeviceToHost, str));
        } else {
            CAV_CUDA(ctx, cudaMemcpyAsync(s.h_out, dp, 4 * m, cudaMemcpyDeviceToHost, str));
            if (t) CAV_CUDA(ctx, cudaMemcpyAsync(s.h_out + 4 * kChunkRays, dt, 4 * m, cudaMemcpyDeviceToHost, str));
            if (uv) CAV_CUDA(ctx, cudaMemcpyAsync(s.h_out + 8 * kChunkRays, duv, 8 * m, cudaMemcpyDeviceToHost, str));
        }
        return CAV_OK;
    };
    auto finish = [&](Slot s, int64_t c) -> cav_status {
        if (out_pinned) return CAV_OK;
        int64_t b = c * kChunkRays, m = std::min(kChunkRays, n - b);
        memcpy(prim_id + b, s.h_out, 4 * m);
        if (t) memcpy(t + b, s.h_out + 4 * kChunkRays, 4 * m);
        if (uv) memcpy(uv + 2 * b, s.h_out + 8 * kChunkRays, 8 * m);
        return CAV_OK;
    };
    return host_pipeline(ctx, n, launch, finish);
}

cav_status cav_trace_any_host(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                              const int32_t* excl_mesh, int64_t n, uint8_t* occluded, uint32_t flags) {
    cav_status st = use_device(ctx);
    if (st != CAV_OK) return st;
    if (!bvh || !rays || !occluded || n < 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_trace_any_host");
    if (n == 0) return CAV_OK;
    const bool in_pinned = is_pinned_host(rays) && (!limit || is_pinned_host(limit)) &&
                           (!excl_mesh || is_pinned_host(excl_mesh));
    const bool out_pinned = is_pinned_host(occluded);
    st = ensure_host_path(ctx, !(in_pinned && out_pinned));
    if (st != CAV_OK) return st;
    st = order_after_build(ctx, bvh);
    if (st != CAV_OK) return st;
    auto launch = [&](Slot s, int64_t c, cudaStream_t str, unsigned long long* counter) -> cav_status {
        int64_t b = c * kChunkRays, m = std::min(kChunkRays, n - b);
        const void* src_r = rays + b;
        const void* src_l = limit ? (const void*)(limit + b) : nullptr;
        const void* src_e = excl_mesh ? (const void*)(excl_mesh + 2 * b) : nullptr;
        if (!in_pinned) {
            memcpy(s.h_rays, rays + b, 32 * m);
            src_r = s.h_rays;
            if (limit) {
                memcpy(s.h_lim, limit + b, 4 * m);
                src_l = s.h_lim;
            }
            if (excl_mesh) {
                memcpy(s.h_excl, excl_mesh + 2 * b, 8 * m);
                src_e = s.h_excl;
            }
        }
        CAV_CUDA(ctx, cudaMemcpyAsync(s.d_rays, src_r, 32 * m, cudaMemcpyHostToDevice, str));
        if (limit) CAV_CUDA(ctx, cudaMemcpyAsync(s.d_lim, src_l, 4 * m, cudaMemcpyHostToDevice, str));
        if (excl_mesh) CAV_CUDA(ctx, cudaMemcpyAsync(s.d_excl, src_e, 8 * m, cudaMemcpyHostToDevice, str));
        uint8_t* docc = (uint8_t*)s.d_out;
        cav_status r = trace_any(ctx, bvh, s.d_rays, limit ? s.d_lim : nullptr, excl_mesh ? s.d_excl : nullptr, m, docc,
                                 flags, str, counter);
        if (r != CAV_OK) return r;
        CAV_CUDA(ctx, cudaMemcpyAsync(out_pinned ? (void*)(occluded + b) : (void*)s.h_out, docc, m,
                                      cudaMemcpyDeviceToHost, str));
        return CAV_OK;
    };
    auto finish = [&](Slot s, int64_t c) -> cav_status {
        if (out_pinned) return CAV_OK;
        int64_t b = c * kChunkRays, m = std::min(kChunkRays, n - b);
        memcpy(occluded + b, s.h_out, m);
        return CAV_OK;
    };
    return host_pipeline(ctx, n, launch, finish);
}

}  // extern "C"
