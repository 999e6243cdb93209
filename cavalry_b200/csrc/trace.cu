// Ray traversal for sm_100a: persistent warps pull 32-ray batches from a device work
// counter, fetch a node (both children's boxes) with four 128-bit read-only loads and
// a triangle with three, and keep the traversal stack in thread-local memory.
//
// Semantics are the reference's BVH::intersect / BVH::testVisibility
// (BVH/BVH.h:23-189): identical slab test (signed-integer min/max on float bit
// patterns, Core/BoundingBox.h:56-74 and Utils/MathsCommons.h:93-100), identical
// Moller-Trumbore test (Core/Triangle.h:7-57), the same child order and the same
// pruning decisions, so hit ids and distances are bit-identical to the reference's
// on the same tree.  The node layout is different: each record holds both children's
// boxes, so one 64-byte fetch replaces the reference's two 44-byte child loads, and
// leaves are folded into their parent's child reference.
#include <cuda_runtime.h>

#include <cfloat>

#include "trace_common.cuh"

namespace cav {

namespace {

// The reference keeps `int stack[64]` without a bound check (BVH/BVH.h:41, :122).  Only
// far children wait on this stack, so it never holds more entries than the tree is deep;
// 128 entries cover the deepest trees the treelet rounds produce on degenerate input, and
// the push is checked (the ray is flagged instead of writing past the end).
constexpr int kStack = 128;
// The short stack is used only for trees whose depth is known to fit: a traversal holds at
// most one deferred sibling per level, so depth + 1 entries always suffice.
constexpr int kShortStack = 64;
// Optionally the first kSmemStack entries of a lane's stack live in shared memory laid out
// [entry][thread]: the 32 lanes of a warp sit in 32 different banks whatever entries they
// touch, so a push or a pop is one L1 wavefront, where in local memory every distinct entry
// among the lanes is its own cache line (ncu on the 1M soup: 4.5 sectors per stack store,
// 7.3 per load, 19 % of the kernel's L1 wavefronts, 77 % of the loads missing L1).  Deeper
// entries stay in local memory.  On the soup 99.85 % of pushes land in the first 16 entries.
constexpr int kSmemStack = 16;

inline size_t stack_smem(int block, int entries) { return sizeof(int32_t) * entries * (size_t)block; }

// With kSmemN == 0 the whole stack is in local memory (the better choice where the
// traversal lives off L1 hits, e.g. coherent rays on a well-built tree: the shared stacks
// shrink the L1); the autotuner times both.
template <int kSmemN>
__device__ __forceinline__ void stack_put(int32_t* sst, int32_t* lst, int i, int32_t v) {
    if (kSmemN > 0 && i < kSmemN) sst[i * (int)blockDim.x] = v;
    else lst[i - kSmemN] = v;
}

template <int kSmemN>
__device__ __forceinline__ int32_t stack_get(const int32_t* sst, const int32_t* lst, int i) {
    return kSmemN > 0 && i < kSmemN ? sst[i * (int)blockDim.x] : lst[i - kSmemN];
}

__device__ inline float imax_f(float a, float b) { return __int_as_float(max(__float_as_int(a), __float_as_int(b))); }
__device__ inline float imin_f(float a, float b) { return __int_as_float(min(__float_as_int(a), __float_as_int(b))); }

// AABB::intersect: returns the entry distance (>= 0) or -1 on a miss.
__device__ inline float slab(float lx, float ly, float lz, float hx, float hy, float hz, const f3& o, const f3& inv) {
    f3 t0 = (mk(lx, ly, lz) - o) * inv;
    f3 t1 = (mk(hx, hy, hz) - o) * inv;
    // fmin_fmax(a,b,c) = int max(int min(a,b), c); fmax_fmin(a,b,c) = int min(int max(a,b), c)
    float maxmin = imax_f(imin_f(t0.x, t1.x), imax_f(imin_f(t0.y, t1.y), fminf(t0.z, t1.z)));
    float minmax = imin_f(imax_f(t0.x, t1.x), imin_f(imax_f(t0.y, t1.y), fmaxf(t0.z, t1.z)));
    if (maxmin <= minmax) {
        if (minmax > 0) return fmaxf(0.f, maxmin);
    }
    return -1.f;
}

// One 64-byte node as two 256-bit read-only loads (sm_100 vector width): each load is one
// 32-byte sector, half the L1 sector lookups of four 16-byte loads.
__device__ __forceinline__ void ld_nc_v8(const void* p, float (&r)[8]) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
                 : "l"(p));
}

struct NodeRegs {
    float lo[8];  // L.lo.xyz L.hi.x L.hi.y L.hi.z R.lo.x R.lo.y
    float hi[8];  // R.lo.z R.hi.xyz left right - -
};

__device__ __forceinline__ void load_node(const TNode* __restrict__ nodes, int32_t ref, NodeRegs& nr) {
    const float* p = reinterpret_cast<const float*>(nodes + ref);
    ld_nc_v8(p, nr.lo);
    ld_nc_v8(p + 8, nr.hi);
}

// Register cap of the single-tree traversal kernels: 48 fit the walk without spills and
// give 42 resident warps per SM where the compiler's own choice (53) gives 36 (measured
// +2.6 % closest-hit rays/s on the 1M soup).  The segmented and instrumented variants
// carry more state and keep 56.  ncu on the soup shows the kernel limited by the L1 data
// pipe's wavefronts (76 % of peak): each lane's node fetch is its own 32-byte wavefront,
// so resident warps matter little and a register-cached stack top or batched triangle
// tests (both tried, both slower) do not pay.
constexpr int kTraceRegs = 48;

// ---------------------------------------------------------------- kernels
// Persistent warps with per-lane ray replacement: every lane owns one ray at a time and
// advances it by one node or one triangle per iteration.  When at least `refill` lanes of a
// warp are idle, the warp claims that many new ray indices from the device work counter
// with one atomic, so lanes whose rays finish early do not wait for the warp's slowest ray.
// Each ray is still traversed exactly as the reference does; only the assignment of rays
// to lanes changes.
// Segments: one traversal launch over the rays of several jobs, each with its own BVH and
// output arrays.  A lane that claims global ray g finds its segment by binary search over
// the segment starts (staged in shared memory) and switches to that segment's tree.
template <bool kCullPop, bool kStats, bool kSeg, int kStackN = kStack, int kSmemN = 0>
__global__ void __maxnreg__(kSeg || kStats ? 56 : kTraceRegs) k_closest(TraceSeg one, const TraceSeg* __restrict__ segs, int nseg, int64_t n,
                          unsigned long long* counter, int refill, uint32_t max_steps, int* flag,
                          unsigned long long* stats) {
    __shared__ int64_t sbeg[kSeg ? kMaxSeg : 1];
    if (kSeg) {
        for (int i = threadIdx.x; i < nseg; i += blockDim.x) sbeg[i] = segs[i].begin;
        __syncthreads();
    }
    if (!kSeg && one.n_dev) n = *one.n_dev;
    const TNode* __restrict__ nodes = one.nodes;
    const TriRec* __restrict__ tris = one.tris;
    float rb0 = 0.f, rb1 = 0.f, rb2 = 0.f, rb3 = 0.f, rb4 = 0.f, rb5 = 0.f;
    if (!kSeg) {
        rb0 = one.root_box[0]; rb1 = one.root_box[1]; rb2 = one.root_box[2];
        rb3 = one.root_box[3]; rb4 = one.root_box[4]; rb5 = one.root_box[5];
    }
    extern __shared__ int32_t sstack[];
    int32_t* const sst = sstack + threadIdx.x;
    int32_t lst[kStackN - kSmemN];
    float sdist[kCullPop ? kStackN : 1];
    TraceStats st;
    bool more = true;
    int64_t ray = -1;  // index within the lane's segment
    int seg = 0;
    f3 o = mk(0, 0, 0), d = mk(0, 0, 0), inv = mk(0, 0, 0);
    float tmax = 0.f, best = 0.f, bu = 0.f, bv = 0.f;
    int32_t bid = -1, ref = 0;
    bool hit = false;
    int top = -1;
    uint32_t steps = 0;
    for (;;) {
        const unsigned idle = __ballot_sync(kFull, ray < 0);
        if (idle == kFull && !more) break;
        if (more && idle != 0 && (__popc(idle) >= refill || idle == kFull)) {
            int64_t r = claim(idle, counter, n, more);
            if (r >= 0) {
                const cav_ray* rays = one.rays;
                if (kSeg) {
                    seg = find_seg(sbeg, nseg, r);
                    const TraceSeg& S = segs[seg];
                    nodes = S.nodes;
                    tris = S.tris;
                    rays = S.rays;
                    r -= S.begin;
                    rb0 = S.root_box[0]; rb1 = S.root_box[1]; rb2 = S.root_box[2];
                    rb3 = S.root_box[3]; rb4 = S.root_box[4]; rb5 = S.root_box[5];
                }
                const float4* rp = reinterpret_cast<const float4*>(rays + r);
                float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
                o = mk(r0.x, r0.y, r0.z);
                d = mk(r1.x, r1.y, r1.z);
                tmax = r1.w;
                inv = mk(1.f / d.x, 1.f / d.y, 1.f / d.z);
                hit = false;
                best = FLT_MAX;
                bu = bv = 0.f;
                bid = -1;
                top = -1;
                ref = 0;
                steps = 0;
                ray = r;
                if (!(slab(rb0, rb1, rb2, rb3, rb4, rb5, o, inv) >= 0.f)) {
                    const TraceSeg& S = kSeg ? segs[seg] : one;
                    S.prim[r] = -1;  // BVH::intersect returns early when the root box is missed
                    if (S.t) S.t[r] = __int_as_float(0x7f800000);
                    if (S.uv) reinterpret_cast<float2*>(S.uv)[r] = make_float2(0.f, 0.f);
                    ray = -1;
                }
            }
        }
        if (ray < 0) continue;
        bool pop = false, overflow = false;
        if (ref >= 0) {
            if (kStats) ++st.nodes;
            NodeRegs nr;
            load_node(nodes, ref, nr);
            const int2 dd = make_int2(__float_as_int(nr.hi[4]), __float_as_int(nr.hi[5]));
            float ml = slab(nr.lo[0], nr.lo[1], nr.lo[2], nr.lo[3], nr.lo[4], nr.lo[5], o, inv);
            float mr = slab(nr.lo[6], nr.lo[7], nr.hi[0], nr.hi[1], nr.hi[2], nr.hi[3], o, inv);
            bool okl = ml >= 0 && ml < best && !(ml > tmax);
            bool okr = mr >= 0 && mr < best && !(mr > tmax);
            if (okl && okr) {
                if (top + 1 >= kStackN) {
                    overflow = true;  // finish below with the flag
                } else {  // the reference pushes the farther child, pops the nearer
                    const bool lfar = ml > mr;
                    ++top;
                    stack_put<kSmemN>(sst, lst, top, lfar ? dd.x : dd.y);
                    if (kCullPop) sdist[top] = lfar ? ml : mr;
                    ref = lfar ? dd.y : dd.x;
                }
            } else if (okl) {
                ref = dd.x;
            } else if (okr) {
                ref = dd.y;
            } else {
                pop = true;
            }
        } else {
            if (kStats) ++st.tris;
            f3 v0, e1, e2;
            int id, mesh;
            load_tri(tris, ~ref, v0, e1, e2, id, mesh);
            float t, u, v;
            if (tri_test(o, d, v0, e1, e2, t, u, v)) {
                if ((!hit || t < best) && !(t > tmax)) {
                    hit = true;
                    best = t;
                    bid = id;
                    bu = u;
                    bv = v;
                }
            }
            pop = true;
        }
        bool finished = false;
        if (overflow || ++steps >= max_steps) {
            atomicOr(flag, overflow ? kFlagStackOverflow : kFlagStepLimit);
            hit = false;
            bid = -2;
            finished = true;
        } else if (pop) {
            if (kCullPop) {
                while (top >= 0 && !(sdist[top] < best)) --top;
            }
            if (top < 0) finished = true;
            else ref = stack_get<kSmemN>(sst, lst, top--);
        }
        if (finished) {
            const TraceSeg& S = kSeg ? segs[seg] : one;
            S.prim[ray] = hit ? bid : (bid == -2 ? -2 : -1);
            if (S.t) S.t[ray] = hit ? best : __int_as_float(0x7f800000);
            if (S.uv) reinterpret_cast<float2*>(S.uv)[ray] = make_float2(bu, bv);
            ray = -1;
        }
    }
    flush_stats<kStats>(st, stats);
}

template <bool kCullPop, bool kStats, bool kSeg, int kStackN = kStack, int kSmemN = 0>
__global__ void __maxnreg__(kSeg || kStats ? 56 : kTraceRegs) k_any(TraceSeg one, const TraceSeg* __restrict__ segs, int nseg, int64_t n,
                      unsigned long long* counter, int refill, uint32_t max_steps, int* flag,
                      unsigned long long* stats) {
    __shared__ int64_t sbeg[kSeg ? kMaxSeg : 1];
    if (kSeg) {
        for (int i = threadIdx.x; i < nseg; i += blockDim.x) sbeg[i] = segs[i].begin;
        __syncthreads();
    }
    if (!kSeg && one.n_dev) n = *one.n_dev;
    const TNode* __restrict__ nodes = one.nodes;
    const TriRec* __restrict__ tris = one.tris;
    extern __shared__ int32_t sstack[];
    int32_t* const sst = sstack + threadIdx.x;
    int32_t lst[kStackN - kSmemN];
    TraceStats st;
    bool more = true;
    int64_t ray = -1;
    int seg = 0;
    f3 o = mk(0, 0, 0), d = mk(0, 0, 0), inv = mk(0, 0, 0);
    float lim = 0.f;
    int32_t src = -1, dst = -1, ref = 0;
    int top = -1;
    uint32_t steps = 0;
    bool use_limit = one.limit != nullptr;
    for (;;) {
        const unsigned idle = __ballot_sync(kFull, ray < 0);
        if (idle == kFull && !more) break;
        if (more && idle != 0 && (__popc(idle) >= refill || idle == kFull)) {
            int64_t r = claim(idle, counter, n, more);
            if (r >= 0) {
                const cav_ray* rays = one.rays;
                const float* limit = one.limit;
                const int32_t* excl = one.excl;
                if (kSeg) {
                    seg = find_seg(sbeg, nseg, r);
                    const TraceSeg& S = segs[seg];
                    nodes = S.nodes;
                    tris = S.tris;
                    rays = S.rays;
                    limit = S.limit;
                    excl = S.excl;
                    use_limit = limit != nullptr;
                    r -= S.begin;
                }
                const float4* rp = reinterpret_cast<const float4*>(rays + r);
                float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
                o = mk(r0.x, r0.y, r0.z);
                d = mk(r1.x, r1.y, r1.z);
                inv = mk(1.f / d.x, 1.f / d.y, 1.f / d.z);
                lim = use_limit ? __ldg(limit + r) : 0.f;
                src = dst = -1;
                if (excl) {
                    int2 e = __ldg(reinterpret_cast<const int2*>(excl) + r);
                    src = e.x;
                    dst = e.y;
                }
                // The reference only reports a root-box miss (BVH/BVH.h:116-120) and traverses anyway.
                top = -1;
                ref = 0;
                steps = 0;
                ray = r;
            }
        }
        if (ray < 0) continue;
        bool pop = false;
        int result = -1;
        if (ref >= 0) {
            if (kStats) ++st.nodes;
            NodeRegs nr;
            load_node(nodes, ref, nr);
            const int2 dd = make_int2(__float_as_int(nr.hi[4]), __float_as_int(nr.hi[5]));
            float ml = slab(nr.lo[0], nr.lo[1], nr.lo[2], nr.lo[3], nr.lo[4], nr.lo[5], o, inv);
            float mr = slab(nr.lo[6], nr.lo[7], nr.hi[0], nr.hi[1], nr.hi[2], nr.hi[3], o, inv);
            bool okl = ml >= 0;
            bool okr = mr >= 0;
            if (kCullPop && use_limit) {
                okl = okl && ml < lim;
                okr = okr && mr < lim;
            }
            if (okl && okr) {
                if (top + 1 >= kStackN) {
                    result = 2;
                    atomicOr(flag, kFlagStackOverflow);
                } else {
                    const bool lfar = ml > mr;
                    stack_put<kSmemN>(sst, lst, ++top, lfar ? dd.x : dd.y);
                    ref = lfar ? dd.y : dd.x;
                }
            } else if (okl) {
                ref = dd.x;
            } else if (okr) {
                ref = dd.y;
            } else {
                pop = true;
            }
        } else {
            if (kStats) ++st.tris;
            f3 v0, e1, e2;
            int id, mesh;
            load_tri(tris, ~ref, v0, e1, e2, id, mesh);
            if (mesh != src && mesh != dst) {
                float t, u, v;
                if (tri_test(o, d, v0, e1, e2, t, u, v)) {
                    if (!use_limit || t < lim) result = 1;
                }
            }
            pop = true;
        }
        if (result < 0 && ++steps >= max_steps) {
            result = 2;
            atomicOr(flag, kFlagStepLimit);
        }
        if (result < 0 && pop) {
            if (top < 0) result = 0;
            else ref = stack_get<kSmemN>(sst, lst, top--);
        }
        if (result >= 0) {
            (kSeg ? segs[seg] : one).occ[ray] = (uint8_t)result;
            ray = -1;
        }
    }
    flush_stats<kStats>(st, stats);
}

// ------------------------------------------------------------------ fast mode (4-wide)
bool use_short_stack(const cav_ctx* ctx, const cav_bvh* bvh) {
    return ctx->trace_stack == kShortStack && bvh->depth >= 0 && bvh->depth + 1 < kShortStack;
}

TraceSeg seg_of(const cav_bvh* bvh) {
    TraceSeg g{};
    g.nodes = bvh->tnodes;
    g.tris = bvh->tris;
    g.root_box = bvh->d_root_box;
    return g;
}

// A persistent traversal launch: the grid fills every SM to the kernel's occupancy with
// `dyn` bytes of shared traversal stacks per block.
template <typename... P, typename... A>
void run_trace(cav_ctx* ctx, void (*kernel)(P...), int block, size_t dyn, cudaStream_t s, A... args) {
    const int grid = grid_for(ctx, kernel, block, dyn);
    kernel<<<grid, block, dyn, s>>>(args...);
}

template <bool kStats, bool kSeg>
cav_status launch_closest(cav_ctx* ctx, const TraceSeg& one, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags,
                          cudaStream_t s, unsigned long long* counter, unsigned long long* stats, bool short_stack = false) {
    const int block = ctx->trace_block > 0 ? ctx->trace_block : 128;
    const int batch = ctx->trace_batch > 0 ? ctx->trace_batch : kDefaultRefill;
    const uint32_t ms = ctx->max_trace_steps;
    int* flag = ctx->d_error + 2;
    CAV_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    const bool plain = !kStats && !kSeg && !(flags & CAV_TRACE_CULL_ON_POP);
    const bool smem = plain && ctx->trace_smem_stack > 0;
    const size_t dyn = smem ? stack_smem(block, kSmemStack) : 0;
    if (plain && short_stack) {
        if (smem)
            run_trace(ctx, k_closest<false, false, false, kShortStack, kSmemStack>, block, dyn, s, one, segs, nseg, n,
                      counter, batch, ms, flag, stats);
        else
            run_trace(ctx, k_closest<false, false, false, kShortStack>, block, dyn, s, one, segs, nseg, n, counter,
                      batch, ms, flag, stats);
    } else if (plain && smem) {
        run_trace(ctx, k_closest<false, false, false, kStack, kSmemStack>, block, dyn, s, one, segs, nseg, n, counter,
                  batch, ms, flag, stats);
    } else if (flags & CAV_TRACE_CULL_ON_POP) {
        run_trace(ctx, k_closest<true, kStats, kSeg>, block, dyn, s, one, segs, nseg, n, counter, batch, ms, flag, stats);
    } else {
        run_trace(ctx, k_closest<false, kStats, kSeg>, block, dyn, s, one, segs, nseg, n, counter, batch, ms, flag, stats);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

template <bool kStats, bool kSeg>
cav_status launch_any(cav_ctx* ctx, const TraceSeg& one, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags,
                      cudaStream_t s, unsigned long long* counter, unsigned long long* stats, bool short_stack = false) {
    const int block = ctx->trace_block > 0 ? ctx->trace_block : 128;
    const int batch = ctx->trace_batch > 0 ? ctx->trace_batch : kDefaultRefill;
    const uint32_t ms = ctx->max_trace_steps;
    int* flag = ctx->d_error + 3;
    CAV_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    const bool plain = !kStats && !kSeg && !(flags & CAV_TRACE_CULL_ON_POP);
    const bool smem = plain && ctx->trace_smem_stack > 0;
    const size_t dyn = smem ? stack_smem(block, kSmemStack) : 0;
    if (plain && short_stack) {
        if (smem)
            run_trace(ctx, k_any<false, false, false, kShortStack, kSmemStack>, block, dyn, s, one, segs, nseg, n,
                      counter, batch, ms, flag, stats);
        else
            run_trace(ctx, k_any<false, false, false, kShortStack>, block, dyn, s, one, segs, nseg, n, counter, batch,
                      ms, flag, stats);
    } else if (plain && smem) {
        run_trace(ctx, k_any<false, false, false, kStack, kSmemStack>, block, dyn, s, one, segs, nseg, n, counter,
                  batch, ms, flag, stats);
    } else if (flags & CAV_TRACE_CULL_ON_POP) {
        run_trace(ctx, k_any<true, kStats, kSeg>, block, dyn, s, one, segs, nseg, n, counter, batch, ms, flag, stats);
    } else {
        run_trace(ctx, k_any<false, kStats, kSeg>, block, dyn, s, one, segs, nseg, n, counter, batch, ms, flag, stats);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

// ---------------------------------------------------------------- ray reordering
// CAV_TRACE_REORDER: a batch is traced in the order of a 30-bit Morton code of its rays'
// origins (normalised to the tree's root box), so the lanes of a warp walk nearby parts of
// the tree and share cache lines; each ray's results go back to its own index.  Every ray is
// traversed on its own, so the hits are those of the given order.  Measured on 4M random
// rays over the 1M-triangle soup: 58.2 ms of traversal against 65.1 in the given order.
constexpr int64_t kReorderMin = (int64_t)1 << 16;  // below this the sort costs more than it saves

__device__ __forceinline__ uint32_t spread10(uint32_t v) {  // bits 0-9 to every third bit
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void k_ray_keys(const cav_ray* __restrict__ rays, int64_t n, const float* __restrict__ box,
                           uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = __ldg(reinterpret_cast<const float4*>(rays + i));
    uint32_t q[3];
    const float oc[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ext = box[3 + a] - box[a];
        const float u = ext > 0.f ? (oc[a] - box[a]) / ext : 0.f;
        q[a] = (uint32_t)fminf(fmaxf(u * 1024.f, 0.f), 1023.f);  // NaN origins clamp to 0
    }
    keys[i] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
    idx[i] = (uint32_t)i;
}

__global__ void k_gather_rays(const cav_ray* __restrict__ rays, const uint32_t* __restrict__ idx, int64_t n,
                              const float* __restrict__ limit, const int32_t* __restrict__ excl, cav_ray* __restrict__ out,
                              float* __restrict__ limit_out, int32_t* __restrict__ excl_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = idx[i];
    const float4* r = reinterpret_cast<const float4*>(rays + j);
    float4* o = reinterpret_cast<float4*>(out + i);
    o[0] = __ldg(r);
    o[1] = __ldg(r + 1);
    if (limit) limit_out[i] = __ldg(limit + j);
    if (excl) reinterpret_cast<int2*>(excl_out)[i] = __ldg(reinterpret_cast<const int2*>(excl) + j);
}

__global__ void k_scatter_closest(const uint32_t* __restrict__ idx, int64_t n, const int32_t* __restrict__ p,
                                  const float* __restrict__ t, const float* __restrict__ uv, int32_t* __restrict__ prim,
                                  float* __restrict__ t_out, float* __restrict__ uv_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = idx[i];
    prim[j] = p[i];
    if (t_out) t_out[j] = t[i];
    if (uv_out) reinterpret_cast<float2*>(uv_out)[j] = reinterpret_cast<const float2*>(uv)[i];
}

__global__ void k_scatter_any(const uint32_t* __restrict__ idx, int64_t n, const uint8_t* __restrict__ o,
                              uint8_t* __restrict__ occ) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    occ[idx[i]] = o[i];
}

// Scratch of one reordered batch: keys and indices (with the sort's second buffers and
// state), the reordered rays and per-ray inputs, and the results in traversal order.
struct ReorderScratch {
    void* base = nullptr;
    uint64_t *keys, *keys_tmp;
    uint32_t *idx, *idx_tmp, *hist, *status, *counters;
    cav_ray* rays;
    float* limit;
    int32_t* excl;
    unsigned char* out;  // 16 bytes per ray
};

cav_status reorder_prepare(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                           const int32_t* excl, int64_t n, cudaStream_t s, ReorderScratch& R) {
    const size_t words = sort_status_words(n, 4);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = (off + bytes + 255) & ~(size_t)255;
        return at;
    };
    const size_t o_keys = take(8 * n), o_keys_tmp = take(8 * n), o_idx = take(4 * n), o_idx_tmp = take(4 * n);
    const size_t o_hist = take(4 * 8 * 256), o_status = take(4 * words), o_counters = take(4 * 4);
    const size_t o_rays = take(32 * n), o_limit = take(limit ? 4 * n : 0), o_excl = take(excl ? 8 * n : 0);
    const size_t o_out = take(16 * n);
    cudaError_t e = dev_alloc(ctx, &R.base, off, s, true);
    if (e != cudaSuccess) return cuda_error(ctx, e, "ray reordering scratch");
    unsigned char* b = (unsigned char*)R.base;
    R.keys = (uint64_t*)(b + o_keys);
    R.keys_tmp = (uint64_t*)(b + o_keys_tmp);
    R.idx = (uint32_t*)(b + o_idx);
    R.idx_tmp = (uint32_t*)(b + o_idx_tmp);
    R.hist = (uint32_t*)(b + o_hist);
    R.status = (uint32_t*)(b + o_status);
    R.counters = (uint32_t*)(b + o_counters);
    R.rays = (cav_ray*)(b + o_rays);
    R.limit = limit ? (float*)(b + o_limit) : nullptr;
    R.excl = excl ? (int32_t*)(b + o_excl) : nullptr;
    R.out = b + o_out;
    const int blocks = (int)div_up(n, 256);
    k_ray_keys<<<blocks, 256, 0, s>>>(rays, n, bvh->d_root_box, R.keys, R.idx);
    cav_status st = sort_pairs(ctx, R.keys, R.idx, R.keys_tmp, R.idx_tmp, n, 4, R.hist, R.status, R.counters,
                               ctx->d_error + 5, s);
    if (st != CAV_OK) {
        cudaFreeAsync(R.base, s);
        return st;
    }
    k_gather_rays<<<blocks, 256, 0, s>>>(rays, R.idx, n, limit, excl, R.rays, R.limit, R.excl);
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

}  // namespace

cav_status trace_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int32_t* prim, float* t,
                         float* uv, uint32_t flags, cudaStream_t s, unsigned long long* counter) {
    if (!bvh || !rays || !prim || n < 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_trace_closest: bad args");
    if (((uintptr_t)rays & 15) != 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
    if (n == 0) return CAV_OK;
    if ((flags & CAV_TRACE_REORDER) && n >= kReorderMin) {
        ReorderScratch R;
        cav_status st = reorder_prepare(ctx, bvh, rays, nullptr, nullptr, n, s, R);
        if (st != CAV_OK) return st;
        int32_t* p = (int32_t*)R.out;
        float* tt = (float*)(R.out + 4 * n);
        float* uu = (float*)(R.out + 8 * n);
        st = trace_closest(ctx, bvh, R.rays, n, p, tt, uu, flags & ~CAV_TRACE_REORDER, s, counter);
        if (st == CAV_OK) {
            k_scatter_closest<<<(unsigned)div_up(n, 256), 256, 0, s>>>(R.idx, n, p, tt, uu, prim, t, uv);
            if (cudaGetLastError() != cudaSuccess) st = set_error(ctx, CAV_ERR_CUDA, "ray reordering scatter");
        }
        cudaFreeAsync(R.base, s);
        return st;
    }
    if (flags & CAV_TRACE_FAST) return trace_wide_closest(ctx, bvh, rays, n, nullptr, prim, t, uv, s, counter);
    TraceSeg one = seg_of(bvh);
    one.rays = rays;
    one.prim = prim;
    one.t = t;
    one.uv = uv;
    return launch_closest<false, false>(ctx, one, nullptr, 0, n, flags, s, counter, nullptr, use_short_stack(ctx, bvh));
}

cav_status trace_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit, const int32_t* excl,
                     int64_t n, uint8_t* occ, uint32_t flags, cudaStream_t s, unsigned long long* counter) {
    if (!bvh || !rays || !occ || n < 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_trace_any: bad args");
    if (((uintptr_t)rays & 15) != 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
    if (excl && ((uintptr_t)excl & 7) != 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "excl must be 8-byte aligned");
    if (n == 0) return CAV_OK;
    if ((flags & CAV_TRACE_REORDER) && n >= kReorderMin) {
        ReorderScratch R;
        cav_status st = reorder_prepare(ctx, bvh, rays, limit, excl, n, s, R);
        if (st != CAV_OK) return st;
        st = trace_any(ctx, bvh, R.rays, R.limit, R.excl, n, R.out, flags & ~CAV_TRACE_REORDER, s, counter);
        if (st == CAV_OK) {
            k_scatter_any<<<(unsigned)div_up(n, 256), 256, 0, s>>>(R.idx, n, R.out, occ);
            if (cudaGetLastError() != cudaSuccess) st = set_error(ctx, CAV_ERR_CUDA, "ray reordering scatter");
        }
        cudaFreeAsync(R.base, s);
        return st;
    }
    if (flags & CAV_TRACE_FAST) return trace_wide_any(ctx, bvh, rays, limit, excl, n, nullptr, occ, s, counter);
    TraceSeg one = seg_of(bvh);
    one.rays = rays;
    one.limit = limit;
    one.excl = excl;
    one.occ = occ;
    return launch_any<false, false>(ctx, one, nullptr, 0, n, flags, s, counter, nullptr, use_short_stack(ctx, bvh));
}

cav_status trace_stats(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                       const float* limit, const int32_t* excl, uint32_t flags, cudaStream_t s, uint64_t* host2) {
    if (!bvh || !rays || n <= 0 || !host2) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_trace_stats: bad args");
    if (((uintptr_t)rays & 15) != 0) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
    void* tmp = nullptr;
    size_t bytes = 64 + (size_t)n * 16;
    CAV_CUDA(ctx, cudaMallocAsync(&tmp, bytes, s));
    unsigned long long* stats = (unsigned long long*)tmp;
    unsigned char* out = (unsigned char*)tmp + 64;
    CAV_CUDA(ctx, cudaMemsetAsync(stats, 0, 16, s));
    cav_status st;
    TraceSeg one = seg_of(bvh);
    one.rays = rays;
    if (flags & CAV_TRACE_FAST) {
        st = any_hit ? trace_wide_any(ctx, bvh, rays, limit, excl, n, nullptr, out, s, ctx->d_counters + 4, stats)
                     : trace_wide_closest(ctx, bvh, rays, n, nullptr, (int32_t*)out, (float*)(out + 4 * n), nullptr, s,
                                          ctx->d_counters + 4, stats);
    } else if (any_hit) {
        one.limit = limit;
        one.excl = excl;
        one.occ = out;
        st = launch_any<true, false>(ctx, one, nullptr, 0, n, flags, s, ctx->d_counters + 4, stats);
    } else {
        one.prim = (int32_t*)out;
        one.t = (float*)(out + 4 * n);
        st = launch_closest<true, false>(ctx, one, nullptr, 0, n, flags, s, ctx->d_counters + 4, stats);
    }
    if (st != CAV_OK) return st;
    unsigned long long h[2];
    CAV_CUDA(ctx, cudaMemcpyAsync(h, stats, 16, cudaMemcpyDeviceToHost, s));
    CAV_CUDA(ctx, cudaFreeAsync(tmp, s));
    CAV_CUDA(ctx, cudaStreamSynchronize(s));
    host2[0] = h[0];
    host2[1] = h[1];
    return CAV_OK;
}

}  // namespace cav

namespace cav {

// One launch over several segments (jobs): segs is a DEVICE array of nseg records whose
// `begin` fields are the prefix sums of their ray counts; n = the total.
cav_status trace_closest_segments(cav_ctx* ctx, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags,
                                  cudaStream_t s, unsigned long long* counter) {
    if (nseg <= 0 || n == 0) return CAV_OK;
    if (nseg > kMaxSeg) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "too many trace segments in one launch");
    if (flags & CAV_TRACE_FAST) return trace_wide_segments(ctx, false, segs, nseg, n, s, counter);
    TraceSeg none{};
    return launch_closest<false, true>(ctx, none, segs, nseg, n, flags, s, counter, nullptr);
}

cav_status trace_any_segments(cav_ctx* ctx, const TraceSeg* segs, int nseg, int64_t n, uint32_t flags, cudaStream_t s,
                              unsigned long long* counter) {
    if (nseg <= 0 || n == 0) return CAV_OK;
    if (nseg > kMaxSeg) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "too many trace segments in one launch");
    if (flags & CAV_TRACE_FAST) return trace_wide_segments(ctx, true, segs, nseg, n, s, counter);
    TraceSeg none{};
    return launch_any<false, true>(ctx, none, segs, nseg, n, flags, s, counter, nullptr);
}

int trace_max_segments() { return kMaxSeg; }

cav_status trace_closest_dev(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const uint32_t* n_dev,
                             int32_t* prim, float* t, float* uv, cudaStream_t s, unsigned long long* counter) {
    TraceSeg one = seg_of(bvh);
    one.rays = rays;
    one.prim = prim;
    one.t = t;
    one.uv = uv;
    one.n_dev = n_dev;
    return launch_closest<false, false>(ctx, one, nullptr, 0, INT64_MAX, CAV_TRACE_EXACT, s, counter, nullptr,
                                        use_short_stack(ctx, bvh));
}

cav_status trace_any_dev(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                         const int32_t* excl, const uint32_t* n_dev, uint8_t* occ, cudaStream_t s,
                         unsigned long long* counter) {
    TraceSeg one = seg_of(bvh);
    one.rays = rays;
    one.limit = limit;
    one.excl = excl;
    one.occ = occ;
    one.n_dev = n_dev;
    return launch_any<false, false>(ctx, one, nullptr, 0, INT64_MAX, CAV_TRACE_EXACT, s, counter, nullptr,
                                    use_short_stack(ctx, bvh));
}

}  // namespace cav

// ================================================================ launch-shape autotuner
// Times the traversal of a ray sample over candidate launch shapes and installs the
// fastest in the context: threads per block, queue chunk (idle lanes before a warp claims
// new rays), and the traversal stack size (the short stack only when the tree's measured
// depth guarantees it cannot overflow).  Blocks per SM stay at the occupancy maximum:
// the kernels are persistent, so fewer resident blocks only idles SMs.
extern "C" cav_status cav_trace_autotune(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, int any_hit,
                                         const float* limit, const int32_t* excl, void* stream,
                                         cav_trace_config_t* best_out) {
    return cav_trace_autotune_flags(ctx, bvh, rays, n, any_hit, limit, excl, CAV_TRACE_EXACT, stream, best_out);
}

// The same search for either traversal mode; the fast (compressed 8-wide) mode has its own
// launch configuration in the context and no stack choice.
extern "C" cav_status cav_trace_autotune_flags(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n,
                                               int any_hit, const float* limit, const int32_t* excl, uint32_t flags,
                                               void* stream, cav_trace_config_t* best_out) {
    using namespace cav;
    if (!ctx || !bvh || !rays || n <= 0) return CAV_ERR_INVALID_ARGUMENT;
    if (flags & ~(uint32_t)(CAV_TRACE_FAST | CAV_TRACE_REORDER)) return CAV_ERR_INVALID_ARGUMENT;
    const bool wide = (flags & CAV_TRACE_FAST) != 0;  // with CAV_TRACE_REORDER every candidate traces the reordered sample
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    if (bvh->depth < 0) {
        int32_t d = 0;
        cav_status st = cav_bvh_depth(ctx, bvh, stream, &d);
        if (st != CAV_OK) return st;
    }
    void* out = nullptr;
    CAV_CUDA(ctx, cudaMallocAsync(&out, (size_t)n * 16 + 256, s));
    int32_t* prim = (int32_t*)out;
    float* t = (float*)((char*)out + 4 * n);
    float* uv = (float*)((char*)out + 8 * n);
    uint8_t* occ = (uint8_t*)out;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int saved[8] = {ctx->trace_block, ctx->trace_blocks_per_sm, ctx->trace_batch, ctx->trace_stack,
                          ctx->wide_block, ctx->wide_batch, ctx->trace_smem_stack, ctx->wide_smem_stack};
    cav_trace_config_t best{0, 0, 0, 0, 1e30f, 0};
    const int blocks[] = {64, 128, 256};
    const int batches[] = {1, 2, 4, 8, 16, 32};
    const int stacks[] = {kStack, kShortStack};
    const int smems[] = {0, wide ? kWideSmemStack : kSmemStack};
    cav_status st = CAV_OK;
    for (int stk : stacks) {
        for (int sm : smems) {
            if (stk == kShortStack && (wide || !(bvh->depth + 1 < kShortStack))) continue;
            for (int blk : blocks)
                for (int bat : batches) {
                    if (wide) {
                        ctx->wide_block = blk;
                        ctx->wide_batch = bat;
                        ctx->wide_smem_stack = sm;
                    } else {
                        ctx->trace_block = blk;
                        ctx->trace_blocks_per_sm = 0;
                        ctx->trace_batch = bat;
                        ctx->trace_stack = stk;
                        ctx->trace_smem_stack = sm;
                    }
                    float ms_best = 1e30f;
                    for (int rep = 0; rep < 3 && st == CAV_OK; ++rep) {  // first repetition warms up
                        cudaEventRecord(a, s);
                        st = any_hit ? trace_any(ctx, bvh, rays, limit, excl, n, occ, flags, s, ctx->d_counters + 5)
                                     : trace_closest(ctx, bvh, rays, n, prim, t, uv, flags, s, ctx->d_counters + 5);
                        cudaEventRecord(b, s);
                        cudaEventSynchronize(b);
                        float ms = 0;
                        cudaEventElapsedTime(&ms, a, b);
                        if (rep > 0) ms_best = std::min(ms_best, ms);
                    }
                    if (st != CAV_OK) break;
                    if (ms_best < best.ms) best = cav_trace_config_t{blk, 0, bat, stk, ms_best, sm};
                }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(out, s);
    if (st != CAV_OK || best.block_threads == 0) {
        ctx->trace_block = saved[0];
        ctx->trace_blocks_per_sm = saved[1];
        ctx->trace_batch = saved[2];
        ctx->trace_stack = saved[3];
        ctx->wide_block = saved[4];
        ctx->wide_batch = saved[5];
        ctx->trace_smem_stack = saved[6];
        ctx->wide_smem_stack = saved[7];
        return st != CAV_OK ? st : set_error(ctx, CAV_ERR_CUDA, "cav_trace_autotune: no candidate ran");
    }
    if (wide) {
        ctx->trace_block = saved[0];  // the exact mode's shape stays as it was
        ctx->trace_blocks_per_sm = saved[1];
        ctx->trace_batch = saved[2];
        ctx->trace_stack = saved[3];
        ctx->trace_smem_stack = saved[6];
        ctx->wide_block = best.block_threads;
        ctx->wide_batch = best.batch;
        ctx->wide_smem_stack = best.smem_stack;
        best.stack = 0;
    } else {
        ctx->trace_block = best.block_threads;
        ctx->trace_blocks_per_sm = 0;
        ctx->trace_batch = best.batch;
        ctx->trace_stack = best.stack;
        ctx->trace_smem_stack = best.smem_stack;
        ctx->wide_block = saved[4];
        ctx->wide_batch = saved[5];
        ctx->wide_smem_stack = saved[7];
    }
    if (best_out) *best_out = best;
    return CAV_OK;
}
