// Treelet restructuring (Karras & Aila 2013) for sm_100a: one warp per treelet root,
// walking bottom-up from the leaves with an arrival counter per node, dynamic
// programming over the 128 leaf subsets staged in shared memory.
//
// Output is bit-identical to the reference's optimizeBVH (BVH/Optimization.cu:467-525
// with optimizeTreelet :49-462): same treelet formation (expand the largest-area
// node, first lane on ties), same partition enumeration order per subset, the same
// warp min-reduction tree for the 6- and 7-leaf subsets, and the same reuse of node
// ids by lane during reconstruction.  It differs in mechanics only:
//   * the warps that start a round are the nodes that are leaves when the round starts,
//     listed by a separate pass (the reference tests `isLeaf` inside the same launch
//     that restructures the tree, Optimization.cu:479);
//   * the formation lanes keep their node records in registers, so every read of the
//     old treelet precedes every write, and the bottom-up box/cost refresh runs on
//     registers with explicit warp synchronisation (the reference iterates 7 times over
//     global memory without __syncwarp, :445-460; its converged values are the same);
//   * subsets of 2..5 leaves are processed grouped by size instead of by the
//     reference's hand-packed 5-round table (each subset's result depends only on the
//     smaller subsets, so the order between subsets does not change any value);
//   * a node whose subtree holds fewer than 7 leaves is not visited by the formation at
//     all (the reference's formation expands such a subtree and gives up without writing);
//   * the walkers are persistent warps that claim their starting leaves from a counter.
#include <cuda_runtime.h>

#include <algorithm>

#include "cav_internal.cuh"

namespace cav {

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct SubsetTable {
    unsigned char s[112];
    int off[5];  // start of popcount 2,3,4,5 and the end
};

constexpr int popc7(int x) { return (x & 1) + ((x >> 1) & 1) + ((x >> 2) & 1) + ((x >> 3) & 1) + ((x >> 4) & 1) + ((x >> 5) & 1) + ((x >> 6) & 1); }

constexpr SubsetTable make_table() {
    SubsetTable t{};
    int k = 0;
    for (int pc = 2; pc <= 5; ++pc) {
        t.off[pc - 2] = k;
        for (int s = 1; s < 128; ++s)
            if (popc7(s) == pc) t.s[k++] = (unsigned char)s;
    }
    t.off[4] = k;
    return t;
}

__constant__ SubsetTable kSubsets = make_table();

struct WarpSmem {
    float area[128];
    float cost[128];
    signed char part[128];
    int leaf_lane[8];
    float lbox[7][6];  // the treelet leaves' boxes (read by every lane: broadcast)
    int32_t lrec[7][4];  // and their left, right, prim, is_leaf
};

struct Rec {
    float lo_x, lo_y, lo_z, hi_x, hi_y, hi_z;
    int32_t left, right, parent, prim;
    float area, cost;
    int32_t is_leaf;
};

__device__ inline Rec load_rec(const BNode* nodes, int32_t id) {
    const float4* p = reinterpret_cast<const float4*>(nodes + id);
    float4 a = __ldcg(p), b = __ldcg(p + 1), c = __ldcg(p + 2), d = __ldcg(p + 3);
    Rec r;
    r.lo_x = a.x; r.lo_y = a.y; r.lo_z = a.z; r.hi_x = a.w;
    r.hi_y = b.x; r.hi_z = b.y; r.left = __float_as_int(b.z); r.right = __float_as_int(b.w);
    r.parent = __float_as_int(c.x); r.prim = __float_as_int(c.y); r.area = c.z; r.cost = c.w;
    r.is_leaf = __float_as_int(d.x);
    return r;
}

__device__ inline void store_rec(BNode* nodes, int32_t id, const Rec& r) {
    float4* p = reinterpret_cast<float4*>(nodes + id);
    __stcg(p, make_float4(r.lo_x, r.lo_y, r.lo_z, r.hi_x));
    __stcg(p + 1, make_float4(r.hi_y, r.hi_z, __int_as_float(r.left), __int_as_float(r.right)));
    __stcg(p + 2, make_float4(__int_as_float(r.parent), __int_as_float(r.prim), r.area, r.cost));
    __stcg(p + 3, make_float4(__int_as_float(r.is_leaf), 0.f, 0.f, 0.f));
}

__device__ inline bool is_pow2(int n) { return (n & (n - 1)) == 0; }

// The reference's warp reduction of partition costs (Optimization.cu:224-266, :271-324): for
// d = 16, 8, 4, 2, 1 lane l takes lane min(l + d, 31)'s candidate when its own is the empty
// -1 or the other is smaller.  Lane 0 ends with the smallest cost; among equal costs with the
// lane whose 5-bit index read backwards is smallest (the bracket keeps the lower lane of
// every pair), and an empty candidate (only lane 0's can be) loses to any other.  Costs are
// non-negative floats, whose bit patterns order like their values, so two min-reductions find
// the same winner; a NaN or negative cost anywhere takes the reference's own loop.  Every lane
// returns lane 0's result.
__device__ inline void reduce_partition(float& tc, int& p) {
    const int lane = threadIdx.x & 31;
    const bool empty = tc == -1.f;
    if (__any_sync(kFull, !empty && !(tc >= 0.f))) {
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
            const int o = min(lane + d, 31);
            const float oc = __shfl_sync(kFull, tc, o);
            const int op = __shfl_sync(kFull, p, o);
            if (tc == -1.f || oc < tc) {
                tc = oc;
                p = op;
            }
        }
        tc = __shfl_sync(kFull, tc, 0);
        p = __shfl_sync(kFull, p, 0);
        return;
    }
    const unsigned key = empty ? 0xffffffffu : __float_as_uint(tc + 0.f);  // +0 for a -0 cost
    const unsigned best = __reduce_min_sync(kFull, key);
    const unsigned rev = __brev((unsigned)lane) >> 27;
    const unsigned win = __brev(__reduce_min_sync(kFull, key == best ? rev : 0xffffffffu)) >> 27;
    tc = __shfl_sync(kFull, tc, (int)win);
    p = __shfl_sync(kFull, p, (int)win);
}

// optimizeTreelet semantics for the subtree rooted at `root`.  Returns false only on
// an internal inconsistency (recorded in *err by the caller).
__device__ bool optimize_treelet(BNode* nodes, int32_t root, int32_t count, WarpSmem& S) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;

    // ---- formation (Optimization.cu:59-107)
    int32_t nid = -1;
    Rec rec{};
    if (lane == 0) {
        nid = root;
        rec = load_rec(nodes, root);
    }
    bool expanded = false;
    int size = 1;
    while (size < 13) {
        // the first of lanes 0..size-1 with the largest area above -1 (lane 0 when none):
        // areas are non-negative, so their bit patterns order like their values
        const bool cand = lane < size && !(rec.is_leaf || expanded) && rec.area > -1.f;
        int max_lane = 0;
        if (__any_sync(kFull, cand && !(rec.area >= 0.f))) {  // a negative area: a plain scan
            float my_area = rec.area;
            if (rec.is_leaf || expanded) my_area = -1.f;
            float max_area = -1.f;
            for (int i = 0; i < size; ++i) {
                float a = __shfl_sync(kFull, my_area, i);
                if (a > max_area) {
                    max_area = a;
                    max_lane = i;
                }
            }
        } else {
            const unsigned key = cand ? __float_as_uint(rec.area + 0.f) + 1u : 0u;
            const unsigned top = __reduce_max_sync(kFull, key);
            if (top != 0u) max_lane = __ffs(__ballot_sync(kFull, key == top)) - 1;
        }
        int stop = __shfl_sync(kFull, (int)(expanded || rec.is_leaf), max_lane);
        if (stop) return true;  // fewer than 7 leaves reachable: leave the subtree as it is
        int32_t cl = __shfl_sync(kFull, rec.left, max_lane);
        int32_t cr = __shfl_sync(kFull, rec.right, max_lane);
        if (cl < 0 || cr < 0 || cl >= count || cr >= count) return false;
        if (lane == max_lane) expanded = true;
        if (lane == size) {
            nid = cl;
            rec = load_rec(nodes, cl);
        }
        if (lane == size + 1) {
            nid = cr;
            rec = load_rec(nodes, cr);
        }
        size += 2;
    }
    const bool in_treelet = lane < 13;
    const unsigned leaf_mask = __ballot_sync(kFull, in_treelet && !expanded);
    const int my_leaf = __popc(leaf_mask & lt);
    if (in_treelet && !expanded) S.leaf_lane[my_leaf] = lane;
    __syncwarp();

    // ---- subset areas (Optimization.cu:126-163)
    // the leaves' records go through shared memory rather than registers (the walk's
    // occupancy is set by its registers)
    if (in_treelet && !expanded) {
        float* b = S.lbox[my_leaf];
        b[0] = rec.lo_x; b[1] = rec.lo_y; b[2] = rec.lo_z;
        b[3] = rec.hi_x; b[4] = rec.hi_y; b[5] = rec.hi_z;
        int32_t* r = S.lrec[my_leaf];
        r[0] = rec.left; r[1] = rec.right; r[2] = rec.prim; r[3] = rec.is_leaf;
    }
    __syncwarp();
    const float(&lbox)[7][6] = S.lbox;
#pragma unroll
    // Subset s = (q << 5) | lane: the union of the lane's leaves 0-4 (its low five bits) is
    // taken once, then leaves 5 and 6 per quarter q (min/max unions are exact in any order).
    bool any = false;
    f3 lo = mk(0, 0, 0), hi = mk(0, 0, 0);
    auto unite = [&](int k, bool& a, f3& l, f3& h) {
        const f3 blo = mk(lbox[k][0], lbox[k][1], lbox[k][2]);
        const f3 bhi = mk(lbox[k][3], lbox[k][4], lbox[k][5]);
        if (!a) {
            l = blo;
            h = bhi;
            a = true;
        } else {
            l = vmin3(l, blo);
            h = vmax3(h, bhi);
        }
    };
#pragma unroll
    for (int k = 0; k < 5; ++k)
        if ((lane >> k) & 1) unite(k, any, lo, hi);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        bool qany = any;
        f3 qlo = lo, qhi = hi;
        if (q & 1) unite(5, qany, qlo, qhi);
        if (q & 2) unite(6, qany, qlo, qhi);
        const int s = (q << 5) | lane;
        S.area[s] = qany ? surface_area(qlo, qhi) : 0.f;
        S.cost[s] = -1.f;
    }
    __syncwarp();
    if (in_treelet && !expanded) S.cost[1 << my_leaf] = rec.cost;
    __syncwarp();

    // ---- subsets of 2..5 leaves (Optimization.cu:180-216), grouped by size
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
        const int b = kSubsets.off[g], e = kSubsets.off[g + 1];
#pragma unroll 1
        for (int k0 = b; k0 < e; k0 += 32) {
            int k = k0 + lane;
            if (k < e) {
                int s = kSubsets.s[k];
                float best = -1.f;
                int bestp = 0;
                int cleared = (s - 1) & s;
                int p = (0 - cleared) & s;
                do {
                    float tc = S.cost[p] + S.cost[s ^ p];
                    if (best == -1.f || tc < best) {
                        bestp = p;
                        best = tc;
                    }
                    p = (p - cleared) & s;
                } while (p != 0);
                S.cost[s] = internal_cost(S.area[s], best);
                S.part[s] = (signed char)bestp;
            }
        }
        __syncwarp();
    }

    // ---- 6-leaf subsets (Optimization.cu:224-266): partition per lane, then the
    // reference's lane-order min reduction (lane l reads lane min(l+d, 31)).
#pragma unroll 1
    for (int eb = 0; eb < 7; ++eb) {
        int s = 0x7f ^ (1 << eb);
        int hi = eb <= 5 ? ((lane << 1) & (((1 << (5 - eb)) - 1) << (eb + 1))) : 0;
        int p = (lane & ((1 << eb) - 1)) | hi;
        float tc = -1.f;
        if (p != 0) tc = S.cost[p] + S.cost[s ^ p];
        reduce_partition(tc, p);
        if (lane == 0) {
            S.cost[s] = internal_cost(S.area[s], tc);
            S.part[s] = (signed char)p;
        }
        __syncwarp();
    }

    // ---- all 7 leaves (Optimization.cu:271-324)
    {
        const int s = 0x7f;
        int p = lane;
        float tc = -1.f;
        if (p != 0) tc = S.cost[p] + S.cost[s ^ p];
        int op = lane | 32;
        float otc = S.cost[op] + S.cost[s ^ op];
        if (tc == -1.f || otc < tc) {
            tc = otc;
            p = op;
        }
        reduce_partition(tc, p);
        if (lane == 0) {
            S.cost[s] = internal_cost(S.area[s], tc);
            S.part[s] = (signed char)p;
        }
        __syncwarp();
    }

    // ---- reconstruction (Optimization.cu:330-394): lane i keeps node nid and takes a role
    int my_subset = lane == 0 ? 0x7f : -1;
    int32_t my_parent = lane == 0 ? rec.parent : -1;
    bool exp_r = false;
    int cl_lane = lane, cr_lane = lane;
    int rsize = 1;
    while (rsize < 13) {
        bool prop = lane < rsize && !exp_r && !is_pow2(my_subset);
        unsigned m = __ballot_sync(kFull, prop);
        if (m == 0) return false;
        int sel_lane = __ffs(m) - 1;
        int sel = __shfl_sync(kFull, my_subset, sel_lane);
        int32_t parent_node = __shfl_sync(kFull, nid, sel_lane);
        int pp = S.part[sel];
        if (sel <= 0 || sel > 127 || is_pow2(sel) || pp <= 0 || (pp & ~sel) != 0) return false;
        if (lane == sel_lane) {
            exp_r = true;
            cl_lane = rsize;
            cr_lane = rsize + 1;
        }
        if (lane == rsize) {
            my_parent = parent_node;
            my_subset = pp;
        }
        if (lane == rsize + 1) {
            my_parent = parent_node;
            my_subset = sel ^ pp;
        }
        rsize += 2;
    }

    // ---- new records (Optimization.cu:400-461)
    int leaf_id = (in_treelet && !exp_r) ? __ffs(my_subset) - 1 : 0;
    Rec o;
    o.lo_x = lbox[leaf_id][0];
    o.lo_y = lbox[leaf_id][1];
    o.lo_z = lbox[leaf_id][2];
    o.hi_x = lbox[leaf_id][3];
    o.hi_y = lbox[leaf_id][4];
    o.hi_z = lbox[leaf_id][5];
    o.left = S.lrec[leaf_id][0];
    o.right = S.lrec[leaf_id][1];
    o.prim = S.lrec[leaf_id][2];
    o.is_leaf = S.lrec[leaf_id][3];
    int32_t child_l = __shfl_sync(kFull, nid, cl_lane);
    int32_t child_r = __shfl_sync(kFull, nid, cr_lane);

    Rec nr;
    nr.parent = my_parent;
    float ocl = 0.f, ocr = 0.f;
    if (!exp_r) {
        nr.lo_x = o.lo_x; nr.lo_y = o.lo_y; nr.lo_z = o.lo_z;
        nr.hi_x = o.hi_x; nr.hi_y = o.hi_y; nr.hi_z = o.hi_z;
        nr.left = o.left;
        nr.right = o.right;
        nr.prim = o.prim;
        nr.is_leaf = o.is_leaf;
        if (in_treelet && !o.is_leaf && o.left >= 0 && o.right >= 0 && o.left < count && o.right < count) {
            ocl = __ldcg(&nodes[o.left].cost);
            ocr = __ldcg(&nodes[o.right].cost);
        }
    } else {
        nr.lo_x = nr.lo_y = nr.lo_z = 0.f;
        nr.hi_x = nr.hi_y = nr.hi_z = 0.f;
        nr.left = child_l;
        nr.right = child_r;
        nr.prim = -1;
        nr.is_leaf = 0;
    }
    // bottom-up boxes: children sit at higher lanes, the treelet is at most 6 deep
#pragma unroll
    for (int it = 0; it < 6; ++it) {
        float a0 = __shfl_sync(kFull, nr.lo_x, cl_lane), b0 = __shfl_sync(kFull, nr.lo_x, cr_lane);
        float a1 = __shfl_sync(kFull, nr.lo_y, cl_lane), b1 = __shfl_sync(kFull, nr.lo_y, cr_lane);
        float a2 = __shfl_sync(kFull, nr.lo_z, cl_lane), b2 = __shfl_sync(kFull, nr.lo_z, cr_lane);
        float a3 = __shfl_sync(kFull, nr.hi_x, cl_lane), b3 = __shfl_sync(kFull, nr.hi_x, cr_lane);
        float a4 = __shfl_sync(kFull, nr.hi_y, cl_lane), b4 = __shfl_sync(kFull, nr.hi_y, cr_lane);
        float a5 = __shfl_sync(kFull, nr.hi_z, cl_lane), b5 = __shfl_sync(kFull, nr.hi_z, cr_lane);
        if (exp_r) {
            f3 lo = vmin3(mk(a0, a1, a2), mk(b0, b1, b2));
            f3 hi = vmax3(mk(a3, a4, a5), mk(b3, b4, b5));
            nr.lo_x = lo.x; nr.lo_y = lo.y; nr.lo_z = lo.z;
            nr.hi_x = hi.x; nr.hi_y = hi.y; nr.hi_z = hi.z;
        }
    }
    nr.area = surface_area(mk(nr.lo_x, nr.lo_y, nr.lo_z), mk(nr.hi_x, nr.hi_y, nr.hi_z));
    if (!exp_r) nr.cost = nr.is_leaf ? leaf_cost(nr.area, 1) : internal_cost(nr.area, ocl, ocr);
    else nr.cost = 0.f;
#pragma unroll
    for (int it = 0; it < 6; ++it) {
        float ca = __shfl_sync(kFull, nr.cost, cl_lane);
        float cb = __shfl_sync(kFull, nr.cost, cr_lane);
        if (exp_r) nr.cost = internal_cost(nr.area, ca, cb);
    }
    if (in_treelet) {
        store_rec(nodes, nid, nr);
        if (!exp_r && !o.is_leaf && o.left >= 0 && o.right >= 0 && o.left < count && o.right < count) {
            __stcg(&nodes[o.left].parent, nid);
            __stcg(&nodes[o.right].parent, nid);
        }
    }
    __syncwarp();
    return true;
}

__global__ void k_leaf_list(const BNode* __restrict__ nodes, int64_t count, int32_t* __restrict__ list,
                            uint32_t* __restrict__ counter) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool leaf = i < count && nodes[i].is_leaf;
    unsigned m = __ballot_sync(kFull, leaf);
    if (m == 0) return;
    int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(kFull, base, __ffs(m) - 1);
    uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
    if (leaf && pos < (uint32_t)((count + 1) / 2)) list[pos] = (int32_t)i;
}

// optimizeBVHImpl (Optimization.cu:467-507): one warp per starting leaf; the second
// arrival at a node optimises the treelet rooted there and continues upwards.
//
// Each walker carries the number of leaves under its node (saturated at 7) in the arrival
// counter: an arrival adds (leaves << 2) | 1, so the second arrival learns its sibling's
// count.  A subtree of fewer than 7 leaves cannot form a treelet: the reference's formation
// then expands every internal node of it and gives up without writing anything (with 7 or
// more leaves an internal node always remains to expand), so such nodes skip formation and
// the tree is unchanged.  The counter's update is an acquire-release atomic: the lanes'
// record writes precede it (warp barrier), and the second arrival's reads follow it.
__device__ void treelet_walk(BNode* nodes, int32_t curr, int32_t count, uint32_t* visited, WarpSmem& S, int* err) {
    const int lane = threadIdx.x & 31;
    if (curr < 0 || curr >= count) {
        if (lane == 0) atomicExch(err, 2);
        return;
    }
    uint32_t leaves = 1;  // under curr, saturated at 7
    for (;;) {
        if (curr == 0) break;
        int32_t parent = __ldcg(&nodes[curr].parent);
        if (parent < 0 || parent >= count) {
            if (lane == 0) atomicExch(err, 2);
            return;
        }
        uint32_t old = 0;
        if (lane == 0)
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                         : "=r"(old)
                         : "l"(visited + parent), "r"((leaves << 2) | 1u)
                         : "memory");
        old = __shfl_sync(kFull, old, 0);
        if ((old & 3u) != 1u) return;  // first arrival stops; the second optimises the parent
        __syncwarp();
        leaves = min(7u, leaves + (old >> 2));
        curr = parent;
        if (leaves >= 7 && !optimize_treelet(nodes, curr, count, S)) {
            if (lane == 0) atomicExch(err, 2);
            return;
        }
        __syncwarp();
    }
}

// Persistent walkers: a fixed grid of 2-warp blocks, 24 per SM (48 warps at 40 registers),
// each warp claiming starting leaves from a counter until the list is exhausted.  The walk
// waits on atomics and dependent loads, so resident walkers matter more than registers,
// and a persistent warp never waits for a block launch after a first arrival ends its walk.
// Measured on 3 rounds over a 1M-triangle soup: one launched warp per leaf in 1-warp blocks
// (32 per SM, 64 registers) 7.14 ms; persistent 1-warp blocks at 64 registers 5.67;
// 2-warp blocks at 48 registers (40 per SM) 5.46; at 40 registers 5.34, 5.00 with the leaf
// boxes in shared memory, 4.93 with the leaf records there too, 4.72 with the subset boxes
// built from per-lane partial unions; at 32 registers (64 per SM) 5.99 (spills).  Claiming
// 4 or 16 leaves per atomic did not help.
constexpr int kWalkWarps = 2;
constexpr int kWalkBlocksPerSm = 24;
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkBlocksPerSm)
    k_treelet(BNode* nodes, const int32_t* __restrict__ list, int64_t n, uint32_t* visited, int* err, uint32_t* claim) {
    __shared__ WarpSmem smem[kWalkWarps];
    WarpSmem& S = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(claim, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= (uint32_t)n) return;
        treelet_walk(nodes, list[i], (int32_t)(2 * n - 1), visited, S, err);
        __syncwarp();
    }
}

// ---- many trees per launch (the batched build): tree k owns leaves [leaf_off[k],
// leaf_off[k+1]) of the concatenated numbering and nodes [2 leaf_off[k] - k, ...) of the
// concatenated node numbering (2 n_k - 1 each).  A launch covers trees [k0, k1); a thread or
// warp finds its tree by binary search over the offsets.
__device__ inline int64_t node_off(const int64_t* leaf_off, int k) { return 2 * leaf_off[k] - k; }

__global__ void k_leaf_list_batch(const TreeletSeg* __restrict__ segs, const int64_t* __restrict__ leaf_off, int k0,
                                  int k1, int32_t* __restrict__ list, uint32_t* __restrict__ counters) {
    const int64_t i = node_off(leaf_off, k0) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < node_off(leaf_off, k1);
    int k = k0;
    int64_t local = 0, n = 0;
    bool leaf = false;
    if (in) {
        int lo = k0, hi = k1 - 1;  // the tree whose node range holds i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (node_off(leaf_off, mid) <= i) lo = mid;
            else hi = mid - 1;
        }
        k = lo;
        local = i - node_off(leaf_off, k);
        n = segs[k].n;
        leaf = local < 2 * n - 1 && segs[k].nodes[local].is_leaf;
    }
    // one atomic per (warp, tree): the lanes of one tree take consecutive list positions in
    // lane order, as the single-tree pass does
    const unsigned leaves = __ballot_sync(kFull, leaf);
    if (!leaf) return;
    const unsigned peers = __match_any_sync(leaves, k) & leaves;
    const int lane = threadIdx.x & 31;
    const int first = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == first) base = atomicAdd(counters + k, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, first);
    const uint32_t pos = base + __popc(peers & ((1u << lane) - 1u));
    if (pos < (uint32_t)n) list[leaf_off[k] + pos] = (int32_t)local;
}

// The same persistent walkers over a group of trees: a claimed index g of the group's
// concatenated leaf list belongs to the tree whose leaf range holds it.
__global__ void __launch_bounds__(kWalkWarps * 32, kWalkBlocksPerSm)
    k_treelet_batch(const TreeletSeg* __restrict__ segs, const int64_t* __restrict__ leaf_off, int k0, int k1,
                    const int32_t* __restrict__ list, uint32_t* visited, int* err, uint32_t* claim) {
    __shared__ WarpSmem smem[kWalkWarps];
    WarpSmem& S = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t first = leaf_off[k0], total = leaf_off[k1] - first;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(claim, 1u);
        i = __shfl_sync(kFull, i, 0);
        if ((int64_t)i >= total) return;
        const int64_t g = first + i;
        int lo = k0, hi = k1 - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (leaf_off[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const int64_t n = segs[lo].n;
        treelet_walk(segs[lo].nodes, list[g], (int32_t)(2 * n - 1), visited + node_off(leaf_off, lo), S, err);
        __syncwarp();
    }
}

}  // namespace

cav_status treelet_rounds(cav_ctx* ctx, BNode* nodes, int64_t n, int rounds, int32_t* leaf_list, uint32_t* visited,
                          uint32_t* counter, cudaStream_t s) {
    if (rounds <= 0) return CAV_OK;
    const int64_t count = 2 * n - 1;
    // counter[0]: the leaf list's positions, counter[1]: the walkers' claims; both in the
    // build's own scratch (builds on different streams, such as a server's lanes, never share it)
    const int64_t grid = std::min<int64_t>(div_up(n, kWalkWarps), (int64_t)ctx->num_sms * kWalkBlocksPerSm);
    for (int r = 0; r < rounds; ++r) {
        CAV_CUDA(ctx, cudaMemsetAsync(visited, 0, sizeof(uint32_t) * count, s));
        CAV_CUDA(ctx, cudaMemsetAsync(counter, 0, 2 * sizeof(uint32_t), s));
        k_leaf_list<<<div_up(count, 256), 256, 0, s>>>(nodes, count, leaf_list, counter);
        k_treelet<<<(unsigned)grid, kWalkWarps * 32, 0, s>>>(nodes, leaf_list, n, visited, ctx->d_error + 1,
                                                             counter + 1);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

// Treelet rounds of K trees, a group of consecutive trees at a time: per group and round one
// leaf-list launch and one treelet launch over all its trees (rather than two per tree).  A
// group holds at most kGroupLeaves leaves; a tree that fills a group alone runs the
// single-tree pass (measured: the grouped kernels were 1.3x slower than it on trees of
// 0.5-2M triangles, and launch overhead does not matter there).  Each tree's result is the
// single-tree one: within a tree the walk is the same, and trees share no nodes.  segs /
// leaf_off: device tables (K trees, K + 1 leaf offsets), segs_host / leaf_off_host the same
// on the host; leaf_list holds leaf_off[K] entries, visited 2 leaf_off[K] - K, counters K + 2
// (per tree leaf-list positions, then the two of a tree that runs the single-tree pass).
cav_status treelet_rounds_batch(cav_ctx* ctx, const TreeletSeg* segs, const TreeletSeg* segs_host,
                                const int64_t* leaf_off, const int64_t* leaf_off_host, int K, int rounds,
                                int32_t* leaf_list, uint32_t* counters, uint32_t* visited, cudaStream_t s) {
    if (rounds <= 0 || K <= 0) return CAV_OK;
    constexpr int64_t kGroupLeaves = (int64_t)1 << 19;
    auto node_off_h = [&](int k) { return 2 * leaf_off_host[k] - k; };
    for (int k0 = 0; k0 < K;) {
        int k1 = k0 + 1;
        while (k1 < K && leaf_off_host[k1 + 1] - leaf_off_host[k0] <= kGroupLeaves) ++k1;
        const int64_t leaves = leaf_off_host[k1] - leaf_off_host[k0];
        const int64_t nodes = node_off_h(k1) - node_off_h(k0);
        if (k1 == k0 + 1 && leaves >= kGroupLeaves / 2) {
            cav_status st = treelet_rounds(ctx, segs_host[k0].nodes, segs_host[k0].n, rounds,
                                           leaf_list + leaf_off_host[k0], visited + node_off_h(k0), counters + K, s);
            if (st != CAV_OK) return st;
            k0 = k1;
            continue;
        }
        const int64_t grid = std::min<int64_t>(div_up(leaves, kWalkWarps), (int64_t)ctx->num_sms * kWalkBlocksPerSm);
        for (int r = 0; r < rounds; ++r) {
            CAV_CUDA(ctx, cudaMemsetAsync(visited + node_off_h(k0), 0, sizeof(uint32_t) * nodes, s));
            CAV_CUDA(ctx, cudaMemsetAsync(counters + k0, 0, sizeof(uint32_t) * (k1 - k0), s));
            CAV_CUDA(ctx, cudaMemsetAsync(counters + K + 1, 0, sizeof(uint32_t), s));  // the walkers' claims
            k_leaf_list_batch<<<div_up(nodes, 256), 256, 0, s>>>(segs, leaf_off, k0, k1, leaf_list, counters);
            k_treelet_batch<<<(unsigned)grid, kWalkWarps * 32, 0, s>>>(segs, leaf_off, k0, k1, leaf_list, visited,
                                                                      ctx->d_error + 1, counters + K + 1);
        }
        k0 = k1;
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

}  // namespace cav
