// Device helpers shared by the traversal kernels (trace.cu: the binary exact mode;
// wide.cu: the compressed 8-wide fast mode): the triangle test, the triangle record load
// and the persistent warps' work claim.
#pragma once

#include "cav_internal.cuh"

namespace cav {

constexpr uint32_t kMaxSteps = 1u << 22;  // default node+triangle visits per ray before the ray is stopped
// Bits of a traversal kind's error word (cav_sync_check maps them to a cav_status).
constexpr int kFlagStackOverflow = 1;  // a push found the traversal stack full
constexpr int kFlagStepLimit = 2;      // a ray reached the context's step limit
constexpr int kDefaultRefill = 4;         // idle lanes that trigger a warp's next claim
// Node groups of the fast mode's stack kept per lane in shared memory when the autotuner
// picks that placement (a lane holds at most one group per wide level).
constexpr int kWideSmemStack = 8;
constexpr unsigned kFull = 0xffffffffu;

// rayTriangleIntersection (Core/Triangle.h:7-57) on precomputed edges.
__device__ inline bool tri_test(const f3& o, const f3& d, const f3& v0, const f3& e1, const f3& e2, float& t, float& u,
                                float& v) {
    f3 tvec = o - v0;
    f3 pvec = cross3(d, e2);
    float det = dot3(e1, pvec);
    if (det == 0) return false;
    det = 1.f / det;
    u = dot3(tvec, pvec) * det;
    if (u < 0.0f || u > 1.0f) return false;
    f3 qvec = cross3(tvec, e1);
    v = dot3(d, qvec) * det;
    if (v < 0.0f || (u + v) > 1.0f) return false;
    t = dot3(e2, qvec) * det;
    if (t <= 0.f) return false;
    return true;
}

__device__ inline void load_tri(const TriRec* __restrict__ tris, int64_t slot, f3& v0, f3& e1, f3& e2, int& id,
                                int& mesh) {
    const float4* p = reinterpret_cast<const float4*>(tris + slot);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    v0 = mk(a.x, a.y, a.z);
    id = __float_as_int(a.w);
    e1 = mk(b.x, b.y, b.z);
    mesh = __float_as_int(b.w);
    e2 = mk(c.x, c.y, c.z);
}

// Claims new rays for the idle lanes of the warp.  Returns the claimed index for this lane
// (or -1) and clears `more` once the counter passed n.
__device__ inline int64_t claim(unsigned idle, unsigned long long* counter, int64_t n, bool& more) {
    const int lane = threadIdx.x & 31;
    const int cnt = __popc(idle);
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, (unsigned long long)cnt);
    base = __shfl_sync(kFull, base, 0);
    if (base + (unsigned long long)cnt >= (unsigned long long)n) more = false;
    if (!((idle >> lane) & 1u)) return -1;
    int64_t my = (int64_t)base + __popc(idle & ((1u << lane) - 1u));
    return my < n ? my : -1;
}

// Segments: one traversal launch over the rays of several jobs, each with its own tree and
// outputs; a lane that claims global ray g finds its segment by binary search over the
// segment starts (staged in shared memory).
constexpr int kMaxSeg = 1024;

__device__ inline int find_seg(const int64_t* sbeg, int nseg, int64_t g) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (sbeg[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Per-lane visit counters of the instrumented traversal variants, summed per warp.
struct TraceStats {
    uint32_t nodes = 0, tris = 0;
};

template <bool kStats>
__device__ inline void flush_stats(const TraceStats& st, unsigned long long* stats) {
    if (!kStats) return;
    unsigned long long a = st.nodes, b = st.tris;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        a += __shfl_down_sync(kFull, a, o);
        b += __shfl_down_sync(kFull, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(stats, a);
        atomicAdd(stats + 1, b);
    }
}

// Blocks of a persistent traversal launch: every SM filled to the kernel's occupancy (or
// the context's configured blocks per SM).
template <typename K>
int grid_for(cav_ctx* ctx, K kernel, int block, size_t dyn_smem = 0) {
    if (dyn_smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
    int per_sm = ctx->trace_blocks_per_sm;
    if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, dyn_smem);
        if (per_sm < 1) per_sm = 1;
    }
    return ctx->num_sms * per_sm;
}

}  // namespace cav
