// The fast traversal mode (CAV_TRACE_FAST): a compressed 8-wide view of the binary tree
// and persistent-warp traversal over it.
//
// Layout (CNode, 80 bytes) after Ylitie, Karras and Laine, "Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs" (HPG 2017): up to eight children per
// node with 8-bit quantised boxes, internal children and triangles each stored
// contiguously, and child slots chosen by direction so that a ray's octant alone gives a
// near-first visiting order.  The view is collapsed from the binary traversal tree
// (TNode) on the device, level by level: a wide node starts from a binary node's two
// children and repeatedly opens the internal child of largest surface area until it has
// eight children or only triangles remain.  Triangles are copied into wide-leaf order so
// that one node's triangles are adjacent in memory.
//
// Traversal keeps a node group (the remaining hit internal children of one node, as a
// bit mask over their visiting order) and a triangle group per ray; only node groups go
// on the stack, 8 bytes each.  A ray visits the same triangles' closest hit as the exact
// mode: the quantised boxes contain the exact ones with a margin, so the closest-hit
// distance is the same and only the choice between triangles at an equal distance may
// differ; the any-hit answer is the same.
#include <cuda_runtime.h>

#include <cfloat>
#include <mutex>

#include "trace_common.cuh"

namespace cav {

namespace {

constexpr int kBuildThreads = 128;
constexpr int kWideStack = 128;       // node groups; one per wide level at most
constexpr int kMaxWideLevels = 4096;  // a wide level consumes at least one binary level
// Relative growth of a box's exit distance, so that the rounding of the two-term plane
// distance never drops a box the ray touches.
constexpr float kGrow = 1.00000095f;  // 1 + 2^-20

__device__ inline void box_of(const TNode& t, int side, float (&b)[6], int32_t& ref) {
    if (side == 0) {
        b[0] = t.a.x; b[1] = t.a.y; b[2] = t.a.z; b[3] = t.a.w; b[4] = t.b.x; b[5] = t.b.y;
        ref = t.d.x;
    } else {
        b[0] = t.b.z; b[1] = t.b.w; b[2] = t.c.x; b[3] = t.c.y; b[4] = t.c.z; b[5] = t.c.w;
        ref = t.d.y;
    }
}

__device__ inline float half_area(const float (&b)[6]) {
    const float ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
    return ex * ey + ey * ez + ez * ex;
}

// One level of the collapse: wide nodes [ctr[2], ctr[3]) each take the binary node task[w].
// ctr[0] counts wide nodes allocated, ctr[1] triangles placed.
__global__ void __launch_bounds__(kBuildThreads)
    k_wide_level(const TNode* __restrict__ tn, const TriRec* __restrict__ tris_in, int32_t* __restrict__ task,
                 CNode* __restrict__ out, TriRec* __restrict__ tris_out, uint32_t* __restrict__ ctr,
                 const float* __restrict__ margin_p) {
    const uint32_t begin = ctr[2], end = ctr[3];
    const float margin = *margin_p;
    for (uint32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x) {
        float cb[8][6];
        int32_t cref[8];
        {
            const TNode t = tn[task[w]];
            box_of(t, 0, cb[0], cref[0]);
            box_of(t, 1, cb[1], cref[1]);
        }
        int cnt = 2;
        while (cnt < 8) {
            int pick = -1;
            float pa = -1.f;
            for (int i = 0; i < cnt; ++i)
                if (cref[i] >= 0) {
                    const float a = half_area(cb[i]);
                    if (a > pa) {
                        pa = a;
                        pick = i;
                    }
                }
            if (pick < 0) break;
            const TNode t = tn[cref[pick]];
            box_of(t, 0, cb[pick], cref[pick]);
            box_of(t, 1, cb[cnt], cref[cnt]);
            ++cnt;
        }
        float lo[3] = {cb[0][0], cb[0][1], cb[0][2]}, hi[3] = {cb[0][3], cb[0][4], cb[0][5]};
        for (int i = 1; i < cnt; ++i)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], cb[i][a]);
                hi[a] = fmaxf(hi[a], cb[i][3 + a]);
            }
        // slots: child i goes to the free slot whose octant diagonal best matches the
        // direction from the node's centre to the child's centre (greedy, largest first)
        float cost[8][8];
        for (int i = 0; i < cnt; ++i) {
            const float cx = (cb[i][0] + cb[i][3]) - (lo[0] + hi[0]);
            const float cy = (cb[i][1] + cb[i][4]) - (lo[1] + hi[1]);
            const float cz = (cb[i][2] + cb[i][5]) - (lo[2] + hi[2]);
            for (int s = 0; s < 8; ++s)
                cost[i][s] = ((s & 4) ? cx : -cx) + ((s & 2) ? cy : -cy) + ((s & 1) ? cz : -cz);
        }
        int slot_child[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        unsigned child_done = 0;
        for (int k = 0; k < cnt; ++k) {
            float bc = -FLT_MAX;
            int bi = -1, bs = -1;
            for (int i = 0; i < cnt; ++i) {
                if (child_done & (1u << i)) continue;
                for (int s = 0; s < 8; ++s)
                    if (slot_child[s] < 0 && (bi < 0 || cost[i][s] > bc)) {
                        bc = cost[i][s];
                        bi = i;
                        bs = s;
                    }
            }
            slot_child[bs] = bi;
            child_done |= 1u << bi;
        }
        // The node's grid: a power-of-two step per axis with 253 steps covering the box grown
        // by the margin, one spare step below it (the origin) and one above.  Every child plane
        // is then rounded outward and moved out by one more step, which absorbs the half-step
        // rounding of the traversal's folded plane distance (node_hits).
        CNode nd;
        float p[3];
        uint32_t ebits = 0;
        double step_inv[3];
        for (int a = 0; a < 3; ++a) {
            const float range = (hi[a] + margin) - (lo[a] - margin);
            int ex = 0;
            frexpf(range * (1.f / 253.f) * 1.0000010f, &ex);  // 2^ex > range / 253
            int eb = ex + 127;
            eb = eb < 1 ? 1 : (eb > 254 ? 254 : eb);
            ebits |= (uint32_t)eb << (8 * a);
            step_inv[a] = ldexp(1.0, 127 - eb);
            p[a] = (lo[a] - margin) - __uint_as_float((uint32_t)eb << 23);
        }
        nd.px = p[0];
        nd.py = p[1];
        nd.pz = p[2];
        int ni = 0, nt = 0;
        for (int i = 0; i < cnt; ++i) (cref[i] >= 0 ? ni : nt) += 1;
        const uint32_t cbase = ni ? atomicAdd(&ctr[0], (uint32_t)ni) : 0u;
        const uint32_t tbase = nt ? atomicAdd(&ctr[1], (uint32_t)nt) : 0u;
        uint32_t imask = 0, meta[2] = {0, 0}, ql[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qh[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        int ri = 0, rt = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = slot_child[s];
            if (i < 0) continue;
            const int word = s >> 2, sh = 8 * (s & 3);
            for (int a = 0; a < 3; ++a) {
                double qlo = floor(((double)cb[i][a] - (double)margin - (double)p[a]) * step_inv[a]) - 1.0;
                double qhi = ceil(((double)cb[i][3 + a] + (double)margin - (double)p[a]) * step_inv[a]) + 1.0;
                qlo = qlo < 0.0 ? 0.0 : (qlo > 255.0 ? 255.0 : qlo);
                qhi = qhi < 0.0 ? 0.0 : (qhi > 255.0 ? 255.0 : qhi);
                ql[a][word] |= (uint32_t)qlo << sh;
                qh[a][word] |= (uint32_t)qhi << sh;
            }
            uint32_t m;
            if (cref[i] >= 0) {
                imask |= 1u << s;
                m = 0x20u | (24u + (uint32_t)s);
                task[cbase + ri] = cref[i];
                ++ri;
            } else {
                m = 0x20u | (uint32_t)rt;
                tris_out[tbase + rt] = tris_in[~cref[i]];
                ++rt;
            }
            meta[word] |= m << sh;
        }
        nd.e_imask = ebits | (imask << 24);
        nd.child_base = cbase;
        nd.tri_base = tbase;
        nd.meta[0] = meta[0];
        nd.meta[1] = meta[1];
        nd.qlo_x[0] = ql[0][0]; nd.qlo_x[1] = ql[0][1];
        nd.qlo_y[0] = ql[1][0]; nd.qlo_y[1] = ql[1][1];
        nd.qlo_z[0] = ql[2][0]; nd.qlo_z[1] = ql[2][1];
        nd.qhi_x[0] = qh[0][0]; nd.qhi_x[1] = qh[0][1];
        nd.qhi_y[0] = qh[1][0]; nd.qhi_y[1] = qh[1][1];
        nd.qhi_z[0] = qh[2][0]; nd.qhi_z[1] = qh[2][1];
        out[w] = nd;
    }
}

__global__ void k_wide_next_level(uint32_t* ctr) {
    if (threadIdx.x == 0) {
        ctr[2] = ctr[3];
        ctr[3] = ctr[0];
    }
}

// Margin of the quantised boxes: 4 ulps of the largest coordinate magnitude of the scene.
__global__ void k_wide_init(const float* root_box, int32_t* task, uint32_t* ctr, float* margin) {
    if (threadIdx.x != 0) return;
    float mag = 0.f;
    for (int k = 0; k < 6; ++k) mag = fmaxf(mag, fabsf(root_box[k]));
    margin[0] = mag * 4.76837158e-7f + 1e-30f;  // 2^-21
    task[0] = 0;  // the binary root becomes wide node 0
    ctr[0] = 1;
    ctr[1] = 0;
    ctr[2] = 0;
    ctr[3] = 1;
}

// ----------------------------------------------------------------------- traversal
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Byte k of w as the float 2^23 + byte (bit pattern 0x4B0000bb).
__device__ __forceinline__ float biased_byte(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | k));
}

struct WideRay {
    f3 o, inv;
    uint32_t octinv4;  // the visiting-order flip (7 - direction octant) in every byte
    bool nx, ny, nz;   // negative direction components
};

// Hit mask of one node: bits 24-31 the internal children in visiting order, bits 0-23 the
// triangles.  `lim` bounds the entry distance (closest hit so far, ray tmax, shadow limit).
// A plane's distance is fma(2^23 + q, s * inv, (p - o) * inv - 2^23 * s * inv): one fma per
// plane on the byte's biased float; the folded constant rounds by at most half a grid step
// in distance, inside the spare step every quantised plane carries.
__device__ __forceinline__ uint32_t node_hits(const CNode* __restrict__ cn, uint32_t idx, const WideRay& R, float lim,
                                              uint32_t& child_base, uint32_t& tri_base, uint32_t& imask) {
    const uint4* q = reinterpret_cast<const uint4*>(cn + idx);
    const uint4 n0 = __ldg(q), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3), n4 = __ldg(q + 4);
    child_base = n1.x;
    tri_base = n1.y;
    imask = n0.w >> 24;
    const float ax = __uint_as_float((n0.w & 0xFFu) << 23) * R.inv.x;
    const float ay = __uint_as_float(((n0.w >> 8) & 0xFFu) << 23) * R.inv.y;
    const float az = __uint_as_float(((n0.w >> 16) & 0xFFu) << 23) * R.inv.z;
    const float bx = (__uint_as_float(n0.x) - R.o.x) * R.inv.x - 8388608.f * ax;
    const float by = (__uint_as_float(n0.y) - R.o.y) * R.inv.y - 8388608.f * ay;
    const float bz = (__uint_as_float(n0.z) - R.o.z) * R.inv.z - 8388608.f * az;
    // near / far planes by direction sign: qlo = (n2.x n2.y | n2.z n2.w | n3.x n3.y), qhi = (n3.z n3.w | n4.x n4.y | n4.z n4.w)
    const uint32_t nx0 = R.nx ? n3.z : n2.x, nx1 = R.nx ? n3.w : n2.y;
    const uint32_t fx0 = R.nx ? n2.x : n3.z, fx1 = R.nx ? n2.y : n3.w;
    const uint32_t ny0 = R.ny ? n4.x : n2.z, ny1 = R.ny ? n4.y : n2.w;
    const uint32_t fy0 = R.ny ? n2.z : n4.x, fy1 = R.ny ? n2.w : n4.y;
    const uint32_t nz0 = R.nz ? n4.z : n3.x, nz1 = R.nz ? n4.w : n3.y;
    const uint32_t fz0 = R.nz ? n3.x : n4.z, fz1 = R.nz ? n3.y : n4.w;
    // per slot byte: the hit bit's position and the bits to set (0 for an empty slot);
    // internal children's positions flip with the ray's octant
    uint32_t bitpos[2], setbits[2];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const uint32_t m4 = w ? n1.w : n1.z;
        const uint32_t inner4 = (((m4 & (m4 << 1)) >> 4) & 0x01010101u) * 0xFFu;  // 0xFF where bits 3 and 4 are set
        bitpos[w] = (m4 ^ (R.octinv4 & inner4)) & 0x1F1F1F1Fu;
        setbits[w] = (m4 >> 5) & 0x07070707u;
    }
    uint32_t hits = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t k = (uint32_t)(i & 3);
        const bool hiw = i >= 4;
        if (hiw && n1.w == 0u) break;  // slots 4-7 empty
        const float tnx = fmaf(biased_byte(hiw ? nx1 : nx0, k), ax, bx);
        const float tny = fmaf(biased_byte(hiw ? ny1 : ny0, k), ay, by);
        const float tnz = fmaf(biased_byte(hiw ? nz1 : nz0, k), az, bz);
        const float tfx = fmaf(biased_byte(hiw ? fx1 : fx0, k), ax, bx);
        const float tfy = fmaf(biased_byte(hiw ? fy1 : fy0, k), ay, by);
        const float tfz = fmaf(biased_byte(hiw ? fz1 : fz0, k), az, bz);
        const float tmin = max3f(tnx, tny, fmaxf(tnz, 0.f));
        const float tmax = fminf(min3f(tfx, tfy, tfz) * kGrow, lim);
        const uint32_t sh = 8u * k;
        const uint32_t bits = tmin <= tmax ? (((hiw ? setbits[1] : setbits[0]) >> sh) & 0xFFu) : 0u;
        hits |= bits << (((hiw ? bitpos[1] : bitpos[0]) >> sh) & 0xFFu);
    }
    return hits;
}

// kSeg: one launch over several jobs' rays (segs[k] = one tree and its outputs, ray indices
// numbered across the launch); otherwise the pointer arguments describe the one tree.
// 64 registers, unconstrained: the kernel is ALU-bound, and capping it for more resident
// warps made the 5.24M-triangle render's extend stage slower (231 ms at 64 registers, 263 at
// 48, 302 at 40).
// The first kSmemN node groups of a lane's stack in shared memory, [entry][thread] (a warp's
// push or pop is two conflict-free wavefronts whatever the lanes' depths), the rest in local
// memory; kSmemN == 0 keeps all of it in local memory.
template <int kSmemN>
__device__ __forceinline__ void wstack_put(uint2* sst, uint2* lst, int i, uint2 v) {
    if (kSmemN > 0 && i < kSmemN) sst[i * (int)blockDim.x] = v;
    else lst[i - kSmemN] = v;
}

template <int kSmemN>
__device__ __forceinline__ uint2 wstack_get(const uint2* sst, const uint2* lst, int i) {
    return kSmemN > 0 && i < kSmemN ? sst[i * (int)blockDim.x] : lst[i - kSmemN];
}

template <bool kAny, bool kStats, bool kSeg, int kSmemN = 0>
__global__ void __launch_bounds__(256)
    k_trace_wide(const CNode* __restrict__ cn0, const TriRec* __restrict__ tris0, const cav_ray* __restrict__ rays0,
                 int64_t n, const uint32_t* n_dev, int32_t* prim0, float* tout0, float* uv0,
                 const float* __restrict__ limit0, const int32_t* __restrict__ excl0, uint8_t* occ0,
                 unsigned long long* counter, int refill, uint32_t max_steps, int* flag,
                 unsigned long long* stats,
                 const TraceSeg* __restrict__ segs, int nseg) {
    __shared__ int64_t sbeg[kSeg ? kMaxSeg : 1];
    if (kSeg) {
        for (int i = threadIdx.x; i < nseg; i += blockDim.x) sbeg[i] = segs[i].begin;
        __syncthreads();
    }
    if (n_dev) n = *n_dev;
    const CNode* __restrict__ cn = cn0;
    const TriRec* __restrict__ tris = tris0;
    int seg = 0;
    TraceStats st;
    extern __shared__ uint2 wsstack[];
    uint2* const sst = wsstack + threadIdx.x;
    uint2 lst[kWideStack - kSmemN];
    bool more = true;
    int64_t ray = -1;
    WideRay R{};
    f3 d = mk(0, 0, 0);
    float tmax = 0.f, best = 0.f, bu = 0.f, bv = 0.f, lim = 0.f;
    int32_t bid = -1, src = -1, dst = -1;
    bool hit = false, use_limit = false;
    uint2 grp = make_uint2(0, 0), tgrp = make_uint2(0, 0);
    int top = -1;
    uint32_t steps = 0;
    for (;;) {
        const unsigned idle = __ballot_sync(kFull, ray < 0);
        if (idle == kFull && !more) break;
        if (more && idle != 0 && (__popc(idle) >= refill || idle == kFull)) {
            int64_t r = claim(idle, counter, n, more);
            if (r >= 0) {
                const cav_ray* rays = rays0;
                const float* limit = limit0;
                const int32_t* excl = excl0;
                if (kSeg) {
                    seg = find_seg(sbeg, nseg, r);
                    const TraceSeg& G = segs[seg];
                    cn = G.cnodes;
                    tris = G.ctris;
                    rays = G.rays;
                    limit = G.limit;
                    excl = G.excl;
                    r -= G.begin;
                }
                const float4* rp = reinterpret_cast<const float4*>(rays + r);
                const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
                R.o = mk(r0.x, r0.y, r0.z);
                d = mk(r1.x, r1.y, r1.z);
                tmax = r1.w;
                // Box tests use a direction whose zero components are replaced by +-2^-66: a
                // finite reciprocal keeps the folded plane distances finite (an infinite one
                // turns them into NaN, which the min / max drop, so the axis would stop
                // bounding the ray and a ray parallel to it would visit a whole slab of the
                // tree).  The triangle test uses the ray's own direction.
                const f3 db = mk(fabsf(d.x) < 1.3552527e-20f ? copysignf(1.3552527e-20f, d.x) : d.x,
                                 fabsf(d.y) < 1.3552527e-20f ? copysignf(1.3552527e-20f, d.y) : d.y,
                                 fabsf(d.z) < 1.3552527e-20f ? copysignf(1.3552527e-20f, d.z) : d.z);
                R.inv = mk(1.f / db.x, 1.f / db.y, 1.f / db.z);
                R.nx = db.x < 0.f;
                R.ny = db.y < 0.f;
                R.nz = db.z < 0.f;
                const uint32_t octinv = 7u - ((R.nx ? 4u : 0u) | (R.ny ? 2u : 0u) | (R.nz ? 1u : 0u));
                R.octinv4 = octinv * 0x01010101u;
                // the root as the one internal child of a virtual parent: slot 0, imask 1
                grp = make_uint2(0u, (1u << (24u + octinv)) | 1u);
                tgrp = make_uint2(0u, 0u);
                hit = false;
                best = FLT_MAX;
                bu = bv = 0.f;
                bid = -1;
                top = -1;
                steps = 0;
                if (kAny) {
                    use_limit = limit != nullptr;
                    lim = use_limit ? __ldg(limit + r) : FLT_MAX;
                    src = dst = -1;
                    if (excl) {
                        const int2 e = __ldg(reinterpret_cast<const int2*>(excl) + r);
                        src = e.x;
                        dst = e.y;
                    }
                }
                ray = r;
            }
        }
        if (ray < 0) continue;
        int result = -1;  // any hit: 0 clear, 1 occluded
        bool finished = false, overflow = false;
        // node phase: a lane without pending triangles takes its next internal child
        if (tgrp.y == 0u) {
            if ((grp.y & 0xFF000000u) == 0u) {
                if (top < 0) {
                    finished = true;
                    result = 0;
                } else {
                    grp = wstack_get<kSmemN>(sst, lst, top--);
                }
            }
            if (!finished) {
                const uint32_t bit = 31u - __clz(grp.y & 0xFF000000u);
                grp.y &= ~(1u << bit);
                const uint32_t slot = (bit - 24u) ^ (R.octinv4 & 7u);
                const uint32_t idx = grp.x + __popc(grp.y & 0xFFu & ((1u << slot) - 1u));
                if (grp.y & 0xFF000000u) {
                    if (top + 1 >= kWideStack) overflow = true;  // flagged below
                    else wstack_put<kSmemN>(sst, lst, ++top, grp);
                }
                uint32_t cbase, tbase, imask;
                const float bound = kAny ? lim : fminf(best, tmax);
                if (kStats) ++st.nodes;
                const uint32_t h = node_hits(cn, idx, R, bound, cbase, tbase, imask);
                grp = make_uint2(cbase, (h & 0xFF000000u) | imask);
                tgrp = make_uint2(tbase, h & 0x00FFFFFFu);
            }
        }
        // triangle phase: one triangle per iteration
        if (!finished && tgrp.y != 0u) {
            const uint32_t k = (uint32_t)(__ffs(tgrp.y) - 1);
            tgrp.y &= tgrp.y - 1u;
            if (kStats) ++st.tris;
            f3 v0, e1, e2;
            int id, mesh;
            load_tri(tris, (int64_t)tgrp.x + k, v0, e1, e2, id, mesh);
            float t, u, v;
            if (kAny) {
                if (mesh != src && mesh != dst && tri_test(R.o, d, v0, e1, e2, t, u, v) && (!use_limit || t < lim)) {
                    result = 1;
                    finished = true;
                }
            } else if (tri_test(R.o, d, v0, e1, e2, t, u, v)) {
                if ((!hit || t < best) && !(t > tmax)) {
                    hit = true;
                    best = t;
                    bid = id;
                    bu = u;
                    bv = v;
                }
            }
        }
        if (!finished && (overflow || ++steps >= max_steps)) {
            atomicOr(flag, overflow ? kFlagStackOverflow : kFlagStepLimit);
            result = 2;
            hit = false;
            bid = -2;
            finished = true;
        }
        if (finished) {
            if (kAny) {
                uint8_t* occ = kSeg ? segs[seg].occ : occ0;
                occ[ray] = (uint8_t)result;
            } else {
                int32_t* prim = kSeg ? segs[seg].prim : prim0;
                float* tout = kSeg ? segs[seg].t : tout0;
                float* uv = kSeg ? segs[seg].uv : uv0;
                prim[ray] = hit ? bid : (bid == -2 ? -2 : -1);
                if (tout) tout[ray] = hit ? best : __int_as_float(0x7f800000);
                if (uv) reinterpret_cast<float2*>(uv)[ray] = make_float2(bu, bv);
            }
            ray = -1;
        }
    }
    flush_stats<kStats>(st, stats);
}

template <bool kAny>
cav_status launch_wide(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, const uint32_t* n_dev,
                       int32_t* prim, float* t, float* uv, const float* limit, const int32_t* excl, uint8_t* occ,
                       cudaStream_t s, unsigned long long* counter, unsigned long long* stats) {
    cav_status st = ensure_wide(ctx, bvh, s);
    if (st != CAV_OK) return st;
    const int block = ctx->wide_block > 0 ? ctx->wide_block : 128;
    const int batch = ctx->wide_batch > 0 ? ctx->wide_batch : kDefaultRefill;
    CAV_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    int* flag = ctx->d_error + (kAny ? 3 : 2);
    if (stats) {
        const int grid = grid_for(ctx, k_trace_wide<kAny, true, false>, block);
        k_trace_wide<kAny, true, false><<<grid, block, 0, s>>>(bvh->cnodes, bvh->ctris, rays, n, n_dev, prim, t, uv,
                                                               limit, excl, occ, counter, batch, ctx->max_trace_steps, flag, stats,
                                                               nullptr, 0);
    } else if (ctx->wide_smem_stack > 0) {
        const size_t dyn = sizeof(uint2) * kWideSmemStack * (size_t)block;
        const int grid = grid_for(ctx, k_trace_wide<kAny, false, false, kWideSmemStack>, block, dyn);
        k_trace_wide<kAny, false, false, kWideSmemStack><<<grid, block, dyn, s>>>(
            bvh->cnodes, bvh->ctris, rays, n, n_dev, prim, t, uv, limit, excl, occ, counter, batch,
            ctx->max_trace_steps, flag, nullptr, nullptr, 0);
    } else {
        const int grid = grid_for(ctx, k_trace_wide<kAny, false, false>, block);
        k_trace_wide<kAny, false, false><<<grid, block, 0, s>>>(bvh->cnodes, bvh->ctris, rays, n, n_dev, prim, t, uv,
                                                                limit, excl, occ, counter, batch, ctx->max_trace_steps,
                                                                flag, nullptr, nullptr, 0);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

}  // namespace

// Several jobs' rays, each against its own tree, in one fast-mode launch (the server's merged
// wavefronts).  Every segment's cnodes / ctris must be set (ensure_wide on its tree).
cav_status trace_wide_segments(cav_ctx* ctx, bool any_hit, const TraceSeg* segs, int nseg, int64_t n, cudaStream_t s,
                               unsigned long long* counter) {
    if (nseg <= 0 || n == 0) return CAV_OK;
    if (nseg > kMaxSeg) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "too many trace segments in one launch");
    const int block = ctx->wide_block > 0 ? ctx->wide_block : 128;
    const int batch = ctx->wide_batch > 0 ? ctx->wide_batch : kDefaultRefill;
    CAV_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    if (any_hit) {
        const int grid = grid_for(ctx, k_trace_wide<true, false, true>, block);
        k_trace_wide<true, false, true><<<grid, block, 0, s>>>(nullptr, nullptr, nullptr, n, nullptr, nullptr, nullptr,
                                                               nullptr, nullptr, nullptr, nullptr, counter, batch,
                                                               ctx->max_trace_steps, ctx->d_error + 3, nullptr, segs,
                                                               nseg);
    } else {
        const int grid = grid_for(ctx, k_trace_wide<false, false, true>, block);
        k_trace_wide<false, false, true><<<grid, block, 0, s>>>(nullptr, nullptr, nullptr, n, nullptr, nullptr, nullptr,
                                                                nullptr, nullptr, nullptr, nullptr, counter, batch,
                                                                ctx->max_trace_steps, ctx->d_error + 2, nullptr, segs,
                                                                nseg);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

cav_status ensure_wide(cav_ctx* ctx, const cav_bvh* bvh, cudaStream_t s) {
    // serialised: several host threads (the server's lanes) may reach one tree at once; the
    // view is published only once its build has completed on the device
    static std::mutex build_mu;
    std::lock_guard<std::mutex> lk(build_mu);
    if (bvh->cnodes) return CAV_OK;
    const int64_t n = bvh->n;
    const int64_t nw = n - 1;  // each wide node but the root stands for a distinct binary internal node
    size_t need = sizeof(CNode) * (size_t)nw + 256;
    need += sizeof(TriRec) * (size_t)n + 256;
    need += sizeof(int32_t) * (size_t)nw + 256;
    need += 64 + 256;
    void* arena = nullptr;  // stream-ordered: complete before the view is published below
    if (dev_alloc(ctx, &arena, need, s, true) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "fast traversal layout: device allocation failed");
    }
    unsigned char* p = (unsigned char*)arena;
    auto carve = [&](size_t bytes) {
        unsigned char* r = (unsigned char*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
        p = r + bytes;
        return (void*)r;
    };
    CNode* cn = (CNode*)carve(sizeof(CNode) * (size_t)nw);
    TriRec* ct = (TriRec*)carve(sizeof(TriRec) * (size_t)n);
    int32_t* task = (int32_t*)carve(sizeof(int32_t) * (size_t)nw);
    uint32_t* ctr = (uint32_t*)carve(32);
    float* margin = (float*)(ctr + 4);
    k_wide_init<<<1, 32, 0, s>>>(bvh->d_root_box, task, ctr, margin);
    const int grid = ctx->num_sms * 8;
    uint32_t* hctr = nullptr;
    if (cudaMallocHost(&hctr, 16) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(arena);
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "fast traversal layout: pinned allocation failed");
    }
    cav_status st = CAV_OK;
    // levels until the frontier is empty; the host looks every 8 levels
    for (int level = 0; level < kMaxWideLevels; ++level) {
        k_wide_level<<<grid, kBuildThreads, 0, s>>>(bvh->tnodes, bvh->tris, task, cn, ct, ctr, margin);
        k_wide_next_level<<<1, 32, 0, s>>>(ctr);
        if ((level & 7) == 7) {
            cudaMemcpyAsync(hctr, ctr, 16, cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                st = cuda_error(ctx, e, "fast traversal layout");
                break;
            }
            if (hctr[2] == hctr[3]) break;
        }
    }
    if (st == CAV_OK) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_error(ctx, e, "fast traversal layout");
        else if (hctr[1] != (uint32_t)n)
            st = set_error(ctx, CAV_ERR_CUDA, "fast traversal layout: not every triangle placed");
    }
    cudaFreeHost(hctr);
    if (st != CAV_OK) {
        cudaFree(arena);
        return st;
    }
    bvh->wide_arena = arena;
    bvh->cnodes = cn;
    bvh->ctris = ct;
    return CAV_OK;
}

void free_wide(cav_bvh* bvh, cudaStream_t s, bool async) {
    if (bvh->wide_arena) {
        if (async) cudaFreeAsync(bvh->wide_arena, s);
        else cudaFree(bvh->wide_arena);
    }
    bvh->wide_arena = nullptr;
    bvh->cnodes = nullptr;
    bvh->ctris = nullptr;
}

cav_status trace_wide_closest(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, int64_t n, const uint32_t* n_dev,
                              int32_t* prim, float* t, float* uv, cudaStream_t s, unsigned long long* counter,
                              unsigned long long* stats) {
    return launch_wide<false>(ctx, bvh, rays, n, n_dev, prim, t, uv, nullptr, nullptr, nullptr, s, counter, stats);
}

cav_status trace_wide_any(cav_ctx* ctx, const cav_bvh* bvh, const cav_ray* rays, const float* limit,
                          const int32_t* excl, int64_t n, const uint32_t* n_dev, uint8_t* occ, cudaStream_t s,
                          unsigned long long* counter, unsigned long long* stats) {
    return launch_wide<true>(ctx, bvh, rays, n, n_dev, nullptr, nullptr, nullptr, limit, excl, occ, s, counter,
                             stats);
}

}  // namespace cav
