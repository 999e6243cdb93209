// LBVH construction for sm_100a: leaf boxes + Morton codes, onesweep radix sort,
// Karras radix tree, fenced atomic bottom-up refit, and the traversal layout.
//
// Semantics follow the reference's BVH::build (BVH/BVH.cu:317-370) so that Morton
// codes, the sorted order and the node array come out bit-identical; the
// implementation is this project's own (see the per-kernel comments for the
// reference lines each one reproduces).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "cav_internal.cuh"

namespace cav {

namespace {

constexpr int kThreads = 256;

// Order-preserving float <-> int32 map for atomic min/max of floats (exact; NaN-free input).
__device__ inline int32_t f2ord(float f) {
    int32_t i = __float_as_int(f);
    return i >= 0 ? i : (i ^ 0x7fffffff);
}
__host__ __device__ inline float ord2f(int32_t i) {
    int32_t b = i >= 0 ? i : (i ^ 0x7fffffff);
#ifdef __CUDA_ARCH__
    return __int_as_float(b);
#else
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}

struct Bounds6 {
    float v[6];
};

// A triangle's three vertex indices, checked against the vertex count.  An index outside
// [0, nv) sets kErrBadIndex and the triangle reads vertex 0 instead, so no load leaves the
// caller's position array (the reference reads whatever the pointer gives).
__device__ inline bool load_tri_idx(const int32_t* __restrict__ idx, int64_t t, int64_t nv, int32_t& a, int32_t& b,
                                    int32_t& c, int* err) {
    a = __ldg(idx + 3 * t);
    b = __ldg(idx + 3 * t + 1);
    c = __ldg(idx + 3 * t + 2);
    if ((uint32_t)a < (uint64_t)nv && (uint32_t)b < (uint64_t)nv && (uint32_t)c < (uint64_t)nv) return true;
    if (err) atomicOr(err, kErrBadIndex);
    a = b = c = 0;
    return false;
}

// Leaf boxes, Core/Triangle.h:242-268 (min/max of the three vertices), written as
// 6 floats per triangle in triangle order, plus an optional scene-bounds reduction
// (the union that Core/Scene.cu:131-135 folds on the host).  A triangle with an index out
// of range gets vertex 0's point box and stays out of the bounds reduction.
__global__ void __launch_bounds__(kThreads) k_leaf_boxes(const float* __restrict__ pos, const int32_t* __restrict__ idx,
                                                         int64_t n, int64_t nv, float* __restrict__ box,
                                                         int32_t* bounds_ord, int* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool valid = i < n;
    if (valid) {
        int32_t a, b, c;
        valid = load_tri_idx(idx, i, nv, a, b, c, err);
        float v0[3], v1[3], v2[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v0[k] = __ldg(pos + 3 * (int64_t)a + k);
            v1[k] = __ldg(pos + 3 * (int64_t)b + k);
            v2[k] = __ldg(pos + 3 * (int64_t)c + k);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(v0[k], fminf(v1[k], v2[k]));
            hi[k] = fmaxf(v0[k], fmaxf(v1[k], v2[k]));
        }
        float* o = box + 6 * i;
        o[0] = lo[0]; o[1] = lo[1]; o[2] = lo[2];
        o[3] = hi[0]; o[4] = hi[1]; o[5] = hi[2];
    }
    if (bounds_ord == nullptr) return;
    // block reduction of the ordered ints
    __shared__ int32_t red[6][kThreads / 32];
    int32_t v[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = valid ? f2ord(lo[k]) : INT32_MAX;
        v[3 + k] = valid ? f2ord(hi[k]) : INT32_MIN;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = __reduce_min_sync(0xffffffffu, v[k]);
        v[3 + k] = __reduce_max_sync(0xffffffffu, v[3 + k]);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) red[k][w] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            int32_t x = l < kThreads / 32 ? red[k][l] : (k < 3 ? INT32_MAX : INT32_MIN);
            x = k < 3 ? __reduce_min_sync(0xffffffffu, x) : __reduce_max_sync(0xffffffffu, x);
            if (l == 0) {
                if (k < 3) atomicMin(bounds_ord + k, x);
                else atomicMax(bounds_ord + k, x);
            }
        }
    }
}

__global__ void k_bounds_init(int32_t* bounds_ord) {
    int k = threadIdx.x;
    if (k < 6) bounds_ord[k] = k < 3 ? INT32_MAX : INT32_MIN;
}

__global__ void k_bounds_decode(const int32_t* bounds_ord, float* bounds) {
    int k = threadIdx.x;
    if (k < 6) bounds[k] = ord2f(bounds_ord[k]);
}

// fillLeafMortonCodes + shiftMorton, BVH/BVH.cu:59-92.  Same expression for the
// normalised centroid (fast-math division, as in the reference) and the same float
// -> uint64 conversion (negative values become 0).  The 21-bit spread is the
// standard 3-D Morton interleave (bit k -> bit 3k); the clamp value 1<<20 is the
// reference's `1 << MORTEN_BITS_PER_DIMENSION - 1`.
__device__ inline uint64_t spread3(uint64_t x) {
    if (x >= (1ull << 21)) x = 1ull << 20;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void __launch_bounds__(kThreads) k_morton(const float* __restrict__ box, int64_t n, const float* dev_bounds,
                                                     Bounds6 host_bounds, int use_dev, uint64_t* __restrict__ codes,
                                                     uint64_t* __restrict__ codes_copy, uint32_t* __restrict__ vals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 slo, shi;
    if (use_dev) {
        slo = mk(dev_bounds[0], dev_bounds[1], dev_bounds[2]);
        shi = mk(dev_bounds[3], dev_bounds[4], dev_bounds[5]);
    } else {
        slo = mk(host_bounds.v[0], host_bounds.v[1], host_bounds.v[2]);
        shi = mk(host_bounds.v[3], host_bounds.v[4], host_bounds.v[5]);
    }
    const float* b = box + 6 * i;
    f3 lo = mk(b[0], b[1], b[2]), hi = mk(b[3], b[4], b[5]);
    f3 centroid = ((lo + hi) * 0.5f - (slo + shi) * 0.5f) / (shi - slo);
    uint64_t factor = (uint64_t)(1L << 21);
    uint64_t x = centroid.x * factor;
    uint64_t y = centroid.y * factor;
    uint64_t z = centroid.z * factor;
    uint64_t code = (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    codes[i] = code;
    codes_copy[i] = code;
    vals[i] = (uint32_t)i;
}

// ------------------------------------------------------------ onesweep sort
// Stable LSD radix sort of 64-bit keys with 32-bit payloads, 8 passes of 8 bits.
// One histogram kernel counts every digit of every pass in a single read; each pass is
// then one kernel: a tile ranks its keys stably (warp match + per-warp counters), and
// finds its global offsets by decoupled look-back over the previous tiles' published
// counts (Merrill & Garland's single-pass prefix scan, as used by Onesweep).
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;

// The histograms of the low `digits` bytes of every key (the digits the sort's passes read),
// in one read of the keys.  Shared counters per block; a warp whose keys share a digit (the
// high digits of spatially coherent primitives) adds them with one atomic, otherwise each
// key adds its own (random digits rarely meet in one warp).
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const uint64_t* __restrict__ keys, int64_t n,
                                                            int digits, uint32_t* __restrict__ hist /*8x256*/) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    // lane 0 of every iterating warp holds a key: i - lane < n
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const bool valid = i < n;
        const uint64_t k = valid ? keys[i] : 0;
        const uint32_t count = __popc(__ballot_sync(0xffffffffu, valid));
        for (int p = 0; p < digits; ++p) {
            const uint32_t d = (uint32_t)(k >> (8 * p)) & 255u;
            const uint32_t d0 = __shfl_sync(0xffffffffu, d, 0);
            if (__all_sync(0xffffffffu, !valid || d == d0)) {
                if (lane == 0) atomicAdd(&h[p][d0], count);
            } else if (valid) {
                atomicAdd(&h[p][d], 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < digits * 256; i += blockDim.x) {
        const uint32_t c = (&h[0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

__device__ inline uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct SortSmem {
    uint64_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t warp_hist[kSortWarps][256];
    uint32_t tile_start[256];
    uint32_t gbase[256];
    uint32_t scan_tmp[256];
    int tile;
};

__global__ void __launch_bounds__(kSortThreads) k_onesweep(const uint64_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin,
                                                           uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                           int64_t n, int shift, const uint32_t* __restrict__ hist,
                                                           uint32_t* status /*tiles x 256*/, uint32_t* tile_counter,
                                                           int* err, uint64_t wait_ns, int stall_first_tile) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) S.tile = (int)atomicAdd(tile_counter, 1u);
    for (int i = tid; i < kSortWarps * 256; i += kSortThreads) (&S.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const int tile = S.tile;
    const int64_t base = (int64_t)tile * kSortTile;

    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
    const int64_t wbase = base + (int64_t)warp * 32 * kSortItems;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t g = wbase + k * 32 + lane;
        bool valid = g < n;
        key[k] = valid ? kin[g] : ~0ull;
        val[k] = valid ? vin[g] : 0u;
    }
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t g = wbase + k * 32 + lane;
        bool valid = g < n;
        uint32_t d = (uint32_t)(key[k] >> shift) & 255u;
        uint32_t peers = __match_any_sync(0xffffffffu, valid ? d : 0x100u);
        int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (valid && lane == leader) {
            old = S.warp_hist[warp][d];
            S.warp_hist[warp][d] = old + (uint32_t)__popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[k] = old + (uint32_t)__popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive offsets across warps and the tile total
    const int digit = tid;  // kSortThreads == 256
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        uint32_t c = S.warp_hist[w][digit];
        S.warp_hist[w][digit] = total;
        total += c;
    }
    // publish this tile's aggregate, then look back for the exclusive prefix
    uint32_t* my_status = status + (size_t)tile * 256 + digit;
    if (tile == 0) {
        // failure injection (tests): the first tile withholds its counts, so every later
        // tile's bounded look-back wait runs out
        if (!stall_first_tile) atomicExch(my_status, kFlagInc | total);
    } else {
        atomicExch(my_status, kFlagAgg | total);
    }
    // Look-back in windows of kLookWin predecessors: their statuses are read at once (one
    // round trip instead of one per tile), then aggregates are summed back to the first
    // inclusive prefix; an entry not yet published is waited on (bounded) and read again.
    // Every tile publishes its aggregate before its own look-back, so the walk back from
    // tile t otherwise takes about t/2 dependent loads.
    constexpr int kLookWin = 8;
    uint32_t excl = 0;
    if (tile > 0) {
        int p = tile - 1;
        uint64_t t0 = 0;
        while (p >= 0) {
            uint32_t st[kLookWin];
#pragma unroll
            for (int w = 0; w < kLookWin; ++w)
                st[w] = p - w >= 0 ? (uint32_t) * ((volatile uint32_t*)(status + (size_t)(p - w) * 256 + digit))
                                   : (uint32_t)kFlagInc;  // before tile 0: an empty inclusive prefix
            int w = 0;
            bool done = false;
#pragma unroll
            for (int k = 0; k < kLookWin; ++k) {
                if (done || w < k) break;  // stopped at an inclusive prefix or an unpublished entry
                const uint32_t f = st[k] & ~kCountMask;
                if (f == 0) break;
                excl += st[k] & kCountMask;
                if (f == kFlagInc) done = true;
                else w = k + 1;
            }
            if (done) break;
            if (w > 0) t0 = 0;  // progress: the wait restarts at the first unpublished entry
            p -= w;
            if (w == kLookWin) continue;
            if (t0 == 0) t0 = globaltimer_ns();
            else if (globaltimer_ns() - t0 > wait_ns) {  // give up and flag the error
                atomicOr(err, kErrLookback);
                break;
            }
        }
        __threadfence();
        atomicExch(my_status, kFlagInc | (excl + total));
    }
    // exclusive scan of tile totals over digits (Hillis-Steele in shared memory)
    S.scan_tmp[digit] = total;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t v = digit >= off ? S.scan_tmp[digit - off] : 0;
        __syncthreads();
        S.scan_tmp[digit] += v;
        __syncthreads();
    }
    uint32_t tstart = S.scan_tmp[digit] - total;
    S.tile_start[digit] = tstart;
    // global exclusive offset of this digit over all keys
    uint32_t h = hist[digit];
    __syncthreads();
    S.scan_tmp[digit] = h;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        uint32_t v = digit >= off ? S.scan_tmp[digit - off] : 0;
        __syncthreads();
        S.scan_tmp[digit] += v;
        __syncthreads();
    }
    S.gbase[digit] = (S.scan_tmp[digit] - h) + excl;
    __syncthreads();
    // scatter into shared memory in tile-sorted order
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        int64_t g = wbase + k * 32 + lane;
        if (g < n) {
            uint32_t d = (uint32_t)(key[k] >> shift) & 255u;
            uint32_t pos = S.tile_start[d] + S.warp_hist[warp][d] + rank[k];
            if (pos < (uint32_t)kSortTile) {
                S.keys[pos] = key[k];
                S.vals[pos] = val[k];
            } else {
                atomicOr(err, kErrSortScatter);
            }
        }
    }
    __syncthreads();
    int64_t tile_n = n - base < kSortTile ? n - base : kSortTile;
    for (int i = tid; i < tile_n; i += kSortThreads) {
        uint64_t k = S.keys[i];
        uint32_t d = (uint32_t)(k >> shift) & 255u;
        uint32_t o = S.gbase[d] + (uint32_t)i - S.tile_start[d];
        if (o < (uint64_t)n) {
            kout[o] = k;
            vout[o] = S.vals[i];
        } else {
            atomicOr(err, kErrSortScatter);
        }
    }
}

// ------------------------------------------------------------- radix tree
// commonPrefixLength, BVH/BVH.cu:101-120, via count-leading-zeros: codes use bits 0..62,
// so differing codes give clz(a^b)-1 equal leading bits; equal codes fall back to
// 63 + the equal leading bits of the 32-bit indices (95 when i == j).
__device__ inline int cpl(const uint64_t* __restrict__ m, uint64_t mi, uint32_t i, uint32_t j) {
    uint64_t mj = __ldg(m + j);
    if (mi != mj) return __clzll((long long)(mi ^ mj)) - 1;
    return 63 + __clz((int)(i ^ j));
}

// buildRadixTree, BVH/BVH.cu:122-215: the same search loops (direction, doubling
// bound, binary search for the other end, the i == 0 override, the float-ceil split
// search, and the `rightChild == leavesCount - 1` leaf clause), writing straight into
// the merged node layout of mergeNodesArray (BVH/BVH.cu:273-302): internal i at i,
// leaf j at N-1+j.
__device__ inline void radix_node(const uint64_t* __restrict__ m, int32_t N, BNode* __restrict__ nodes, int32_t i,
                                  int* err) {
    const uint64_t mi = __ldg(m + i);
    int d = 1;
    if (i > 0) d = (cpl(m, mi, i, i + 1) - cpl(m, mi, i, i - 1)) >= 0 ? 1 : -1;
    int minCPL = 0;
    if (i > 0) minCPL = cpl(m, mi, i, (uint32_t)(i - d));
    uint32_t maxLength = 2;
    for (;;) {
        int64_t jj = (int64_t)i + (int64_t)maxLength * d;
        if (!(jj >= 0 && jj < N)) break;
        if (!(cpl(m, mi, i, (uint32_t)jj) > minCPL)) break;
        maxLength *= 2;
    }
    uint32_t length = 0;
    for (int power = 1;; ++power) {
        uint32_t t = maxLength >> power;
        if (t == 0) break;
        int32_t j = (int32_t)((uint32_t)i + (length + t) * (uint32_t)d);
        if (j >= 0 && j < N && cpl(m, mi, i, j) > minCPL) length += t;
    }
    int32_t j = (int32_t)((uint32_t)i + length * (uint32_t)d);
    if (i == 0) j = N - 1;
    int prefix = cpl(m, mi, i, j);
    uint32_t dist = 0;
    for (int power = 1;; ++power) {
        uint32_t t = ceil((float)length / ((float)(1 << power)));
        int32_t jj = (int32_t)((uint32_t)i + (dist + t) * (uint32_t)d);
        if (jj >= 0 && jj < N && cpl(m, mi, i, jj) > prefix) dist += t;
        if (t <= 1) break;
    }
    int32_t split = (int32_t)((uint32_t)i + dist * (uint32_t)d) + min(0, d);
    int32_t lc = split, rc = split + 1;
    if (lc < 0 || rc > N - 1) {
        atomicOr(err, kErrRadixSplit);
        return;
    }
    bool lleaf = min(i, j) == lc;
    bool rleaf = (max(i, j) == rc) || (rc == N - 1);
    int32_t lid = lleaf ? N - 1 + lc : lc;
    int32_t rid = rleaf ? N - 1 + rc : rc;
    BNode& nd = nodes[i];
    nd.left = lid;
    nd.right = rid;
    nd.prim = -1;
    nd.is_leaf = 0;
    nodes[lid].parent = i;
    nodes[rid].parent = i;
    if (i == 0) nd.parent = 0;  // GpuArray zero fill: the root's parent field reads 0
}

__global__ void __launch_bounds__(kThreads) k_radix_tree(const uint64_t* __restrict__ m, int32_t N,
                                                         BNode* __restrict__ nodes, int* err) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N - 1) return;
    radix_node(m, N, nodes, i, err);
}

// Leaf records (fillLeafBoundingBoxes + copyLeafNode, BVH/BVH.cu:46-56, 261-271) and
// computeBounds (BVH/BVH.cu:217-259): the second arrival at a node unions its
// children.  Child records written by other threads are read through L2 (ld.cg)
// after an acquire fence; writes are published with a release fence before the
// arrival counter is bumped (the reference has no fence here).
// box_index: the leaf's triangle in `box`; prim: the triangle id the leaf records
__device__ inline void refit_leaf(const float* __restrict__ box, uint32_t box_index, int32_t prim, int32_t N,
                                  BNode* nodes, uint32_t* visited, int32_t j, int* err) {
    const uint32_t t = box_index;
    const float* b = box + 6 * (size_t)t;
    f3 lo = mk(b[0], b[1], b[2]), hi = mk(b[3], b[4], b[5]);
    BNode* L = nodes + (N - 1 + j);
    L->lo_x = lo.x; L->lo_y = lo.y; L->lo_z = lo.z;
    L->hi_x = hi.x; L->hi_y = hi.y; L->hi_z = hi.z;
    L->left = 0;
    L->right = 0;
    L->prim = prim;
    L->is_leaf = 1;
    float area = surface_area(lo, hi);
    L->area = area;
    L->cost = leaf_cost(area, 1);
    __threadfence();
    int32_t curr = L->parent;
    for (;;) {
        if (curr < 0 || curr >= N - 1) {
            atomicOr(err, kErrRefitLink);
            return;
        }
        uint32_t old = atomicAdd(visited + curr, 1u);
        if (old != 1) return;  // first arrival (or a malformed third) stops here
        __threadfence();
        BNode* nd = nodes + curr;
        int32_t l = __ldcg(&nd->left), r = __ldcg(&nd->right);
        if (l < 0 || r < 0 || l >= 2 * N - 1 || r >= 2 * N - 1) {
            atomicOr(err, kErrRefitLink);
            return;
        }
        const BNode* A = nodes + l;
        const BNode* B = nodes + r;
        f3 alo = mk(__ldcg(&A->lo_x), __ldcg(&A->lo_y), __ldcg(&A->lo_z));
        f3 ahi = mk(__ldcg(&A->hi_x), __ldcg(&A->hi_y), __ldcg(&A->hi_z));
        f3 blo = mk(__ldcg(&B->lo_x), __ldcg(&B->lo_y), __ldcg(&B->lo_z));
        f3 bhi = mk(__ldcg(&B->hi_x), __ldcg(&B->hi_y), __ldcg(&B->hi_z));
        float cl = __ldcg(&A->cost), cr = __ldcg(&B->cost);
        f3 nlo = vmin3(alo, blo), nhi = vmax3(ahi, bhi);
        nd->lo_x = nlo.x; nd->lo_y = nlo.y; nd->lo_z = nlo.z;
        nd->hi_x = nhi.x; nd->hi_y = nhi.y; nd->hi_z = nhi.z;
        float a = surface_area(nlo, nhi);
        nd->area = a;
        nd->cost = internal_cost(a, cl, cr);
        __threadfence();
        if (curr == 0) return;
        curr = __ldcg(&nd->parent);
    }
}

__global__ void __launch_bounds__(kThreads) k_refit(const float* __restrict__ box, const uint32_t* __restrict__ perm,
                                                    int32_t N, BNode* nodes, uint32_t* visited, int* err) {
    int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    const uint32_t t = perm[j];
    if (t >= (uint32_t)N) {  // a permutation entry out of range (after a failed sort)
        atomicOr(err, kErrRefitLink);
        return;
    }
    refit_leaf(box, t, (int32_t)t, N, nodes, visited, j, err);
}

// ---------------------------------------------------------------- layout
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ inline uint32_t block_excl_scan(uint32_t v, uint32_t* wsum, uint32_t* total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    uint32_t before = w > 0 ? wsum[w - 1] : 0;
    if (total) *total = wsum[(blockDim.x >> 5) - 1];
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_count_internal(const BNode* __restrict__ nodes, int64_t count,
                                                                 uint32_t* __restrict__ block_counts) {
    __shared__ uint32_t wsum[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < count && !nodes[base + k].is_leaf) ++c;
    uint32_t total;
    block_excl_scan(c, wsum, &total);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(uint32_t* counts, int nblocks) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += kScanThreads) {
        int b = b0 + threadIdx.x;
        uint32_t v = b < nblocks ? counts[b] : 0;
        uint32_t total;
        uint32_t e = block_excl_scan(v, wsum, &total);
        if (b < nblocks) counts[b] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads) k_compact_index(const BNode* __restrict__ nodes, int64_t count,
                                                                const uint32_t* __restrict__ block_offsets,
                                                                int32_t* __restrict__ compact) {
    __shared__ uint32_t wsum[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    bool in[kScanItems];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        in[k] = base + k < count && !nodes[base + k].is_leaf;
        c += in[k];
    }
    uint32_t e = block_excl_scan(c, wsum, nullptr) + block_offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < count) compact[base + k] = in[k] ? (int32_t)(e++) : -1;
    }
}

// Triangle records in sorted (Morton) order; slot_of[t] = sorted position of triangle t.
__global__ void __launch_bounds__(kThreads) k_tri_layout(const float* __restrict__ pos, int64_t nv,
                                                         const int32_t* __restrict__ idx,
                                                         const int32_t* __restrict__ mesh, const uint32_t* __restrict__ perm,
                                                         int64_t n, TriRec* __restrict__ tris, int32_t* __restrict__ slot_of) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t t = perm[j];
    if (t >= (uint64_t)n) t = 0;  // a permutation entry out of range (a failed sort, flagged there)
    int32_t a, b, c;
    load_tri_idx(idx, t, nv, a, b, c, nullptr);  // already flagged by the leaf-box pass
    f3 v0 = mk(pos[3 * (size_t)a], pos[3 * (size_t)a + 1], pos[3 * (size_t)a + 2]);
    f3 v1 = mk(pos[3 * (size_t)b], pos[3 * (size_t)b + 1], pos[3 * (size_t)b + 2]);
    f3 v2 = mk(pos[3 * (size_t)c], pos[3 * (size_t)c + 1], pos[3 * (size_t)c + 2]);
    f3 e1 = v1 - v0, e2 = v2 - v0;
    int32_t m = mesh ? mesh[t] : 0;
    TriRec r;
    r.v0 = make_float4(v0.x, v0.y, v0.z, __int_as_float((int)t));
    r.e1 = make_float4(e1.x, e1.y, e1.z, __int_as_float(m));
    r.e2 = make_float4(e2.x, e2.y, e2.z, 0.f);
    tris[j] = r;
    slot_of[t] = (int32_t)j;
}

__global__ void __launch_bounds__(kThreads) k_tnode_layout(const BNode* __restrict__ nodes, int64_t count,
                                                           const int32_t* __restrict__ compact,
                                                           const int32_t* __restrict__ slot_of,
                                                           TNode* __restrict__ out, float* __restrict__ root_box) {
    int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= count) return;
    const BNode& nd = nodes[x];
    if (x == 0) {
        root_box[0] = nd.lo_x; root_box[1] = nd.lo_y; root_box[2] = nd.lo_z;
        root_box[3] = nd.hi_x; root_box[4] = nd.hi_y; root_box[5] = nd.hi_z;
    }
    if (nd.is_leaf) return;
    if (nd.left < 0 || nd.left >= count || nd.right < 0 || nd.right >= count) return;  // a failed build
    const BNode& A = nodes[nd.left];
    const BNode& B = nodes[nd.right];
    const int64_t n = (count + 1) / 2;
    const bool lp = A.prim >= 0 && A.prim < n, rp = B.prim >= 0 && B.prim < n;
    int32_t lref = A.is_leaf ? ~(lp ? slot_of[A.prim] : 0) : compact[nd.left];
    int32_t rref = B.is_leaf ? ~(rp ? slot_of[B.prim] : 0) : compact[nd.right];
    int32_t c = compact[x];
    if (c < 0 || c >= count / 2) return;  // N-1 internal slots
    TNode t;
    t.a = make_float4(A.lo_x, A.lo_y, A.lo_z, A.hi_x);
    t.b = make_float4(A.hi_y, A.hi_z, B.lo_x, B.lo_y);
    t.c = make_float4(B.lo_z, B.hi_x, B.hi_y, B.hi_z);
    t.d = make_int4(lref, rref, 0, 0);
    out[c] = t;
}

__global__ void k_merge_error(const int* src, int* dst) {
    if (threadIdx.x == 0 && src[0] != 0) atomicOr(dst, src[0]);
}

// After a structural build error (kErrStructural): node 0 of the traversal layout points
// both children at triangle slot 0, which becomes an all-zero record that every triangle test
// rejects (zero determinant), so a tree whose build failed is still safe to trace and
// reports no hits; cav_sync_check reports the error.
__global__ void k_poison_tree(const int* err, TNode* tnodes, TriRec* tris) {
    if (threadIdx.x != 0 || !(*err & kErrStructural)) return;
    TNode t;
    t.a = t.b = t.c = make_float4(0.f, 0.f, 0.f, 0.f);
    t.d = make_int4(~0, ~0, 0, 0);
    tnodes[0] = t;
    TriRec r;
    r.v0 = r.e1 = r.e2 = make_float4(0.f, 0.f, 0.f, 0.f);
    tris[0] = r;
}

template <typename T>
T* carve(unsigned char*& p, size_t count) {
    size_t off = ((uintptr_t)p + 255) & ~(uintptr_t)255;
    T* r = reinterpret_cast<T*>(off);
    p = reinterpret_cast<unsigned char*>(off + sizeof(T) * count);
    return r;
}

}  // namespace

// The persistent arrays of one tree (build nodes, codes, permutation, traversal layout),
// carved from `base`, which must hold bvh_arena_bytes(n).
size_t bvh_arena_bytes(int64_t n) {
    const int64_t count = 2 * n - 1;
    size_t need = 0;
    need += sizeof(BNode) * count + 256;
    need += 2 * (sizeof(uint64_t) * n + 256);
    need += sizeof(int32_t) * n + 256;
    need += sizeof(TNode) * (n - 1) + 256;
    need += sizeof(TriRec) * n + 256;
    need += 64 + 256;
    return need;
}

static cav_bvh* carve_bvh(cav_ctx* ctx, int64_t n, unsigned char* base) {
    const int64_t count = 2 * n - 1;
    cav_bvh* bvh = new cav_bvh();
    bvh->n = n;
    bvh->device = ctx->device;
    unsigned char* p = base;
    bvh->nodes = carve<BNode>(p, count);
    bvh->codes_unsorted = carve<uint64_t>(p, n);
    bvh->codes_sorted = carve<uint64_t>(p, n);
    bvh->perm = carve<int32_t>(p, n);
    bvh->tnodes = carve<TNode>(p, n - 1);
    bvh->tris = carve<TriRec>(p, n);
    bvh->d_root_box = carve<float>(p, 8);
    bvh->d_depth = carve<int32_t>(p, 8);
    return bvh;
}

// One tree's arena, stream-ordered on the build's stream (the tree is used there first).
cav_status alloc_bvh(cav_ctx* ctx, int64_t n, cudaStream_t s, cav_bvh** out) {
    void* arena = nullptr;
    if (dev_alloc(ctx, &arena, bvh_arena_bytes(n), s, true) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "cav_bvh_build: device allocation failed");
    }
    cav_bvh* bvh = carve_bvh(ctx, n, (unsigned char*)arena);
    bvh->arena = arena;
    *out = bvh;
    return CAV_OK;
}

// Releases a tree: its events, its fast-mode view and its arena (or its share of a batch's
// arena, freed with the last tree of the batch).  async: stream-ordered frees on `s`.
void bvh_release(cav_bvh* bvh, cudaStream_t s, bool async) {
    if (!bvh) return;
    if (bvh->timed)
        for (int k = 0; k < 7; ++k) cudaEventDestroy(bvh->ev[k]);
    free_wide(bvh, s, async);
    void* mem = bvh->arena;
    if (bvh->shared) {
        mem = nullptr;
        if (bvh->shared->refs.fetch_sub(1) == 1) {
            mem = bvh->shared->p;
            delete bvh->shared;
        }
    }
    if (mem) {
        if (async) cudaFreeAsync(mem, s);
        else cudaFree(mem);
    }
    delete bvh;
}

cav_status build_bvh(cav_ctx* ctx, const float* positions, int64_t nv, const int32_t* indices,
                     const int32_t* mesh_ids, int64_t n, const float* bounds, int rounds, cudaStream_t s,
                     cav_bvh** out) {
    if (!positions || !indices || !out || nv < 1 || n < 2 || n >= (1ll << 30) || rounds < 0)
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_build: invalid argument");
    const int64_t count = 2 * n - 1;
    cav_bvh* bvh = nullptr;
    cav_status ast = alloc_bvh(ctx, n, s, &bvh);
    if (ast != CAV_OK) return ast;

    // scratch (stream ordered)
    const int tiles = div_up(n, kSortTile);
    size_t scratch = 0;
    scratch += sizeof(float) * 6 * n + 256;           // leaf boxes
    scratch += sizeof(uint64_t) * n + 256;            // sort ping-pong keys
    scratch += sizeof(uint32_t) * n + 256;            // sort vals A
    scratch += sizeof(uint32_t) * n + 256;            // sort vals B
    scratch += sizeof(uint32_t) * 8 * 256 + 256;      // histograms
    scratch += sizeof(uint32_t) * 8 * (size_t)tiles * 256 + 256;  // look-back status
    scratch += sizeof(uint32_t) * 16 + 256;           // tile counters + bounds ords
    scratch += sizeof(int32_t) * 8 + 256;             // error flag
    scratch += sizeof(float) * 8 + 256;               // device bounds
    scratch += sizeof(uint32_t) * count + 256;        // visited
    scratch += sizeof(int32_t) * n + 256;             // leaf list
    scratch += sizeof(int32_t) * count + 256;         // compact index
    scratch += sizeof(int32_t) * n + 256;             // slot_of
    scratch += sizeof(uint32_t) * (div_up(count, kScanTile) + 1) + 256;
    void* sbase = nullptr;
    cudaError_t e = dev_alloc(ctx, &sbase, scratch, s, true);
    if (e != cudaSuccess) {
        cudaGetLastError();
        bvh_release(bvh, s, true);
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "cav_bvh_build: scratch allocation failed");
    }
    unsigned char* q = (unsigned char*)sbase;
    float* leafbox = carve<float>(q, 6 * n);
    uint64_t* keys_b = carve<uint64_t>(q, n);
    uint32_t* vals_a = carve<uint32_t>(q, n);
    uint32_t* vals_b = carve<uint32_t>(q, n);
    uint32_t* hist = carve<uint32_t>(q, 8 * 256);
    uint32_t* status = carve<uint32_t>(q, 8 * (size_t)tiles * 256);
    uint32_t* counters = carve<uint32_t>(q, 16);  // [0..7] tile counters, [8..13] bounds ords, [14..15] treelets
    int32_t* err = carve<int32_t>(q, 8);
    float* dbounds = carve<float>(q, 8);
    uint32_t* visited = carve<uint32_t>(q, count);
    int32_t* leaf_list = carve<int32_t>(q, n);
    int32_t* compact = carve<int32_t>(q, count);
    int32_t* slot_of = carve<int32_t>(q, n);
    uint32_t* blk = carve<uint32_t>(q, div_up(count, kScanTile) + 1);

    for (int k = 0; k < 7; ++k) cudaEventCreate(&bvh->ev[k]);
    bvh->timed = true;

    CAV_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, s));
    CAV_CUDA(ctx, cudaMemsetAsync(status, 0, sizeof(uint32_t) * 8 * (size_t)tiles * 256, s));
    CAV_CUDA(ctx, cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 16, s));
    CAV_CUDA(ctx, cudaMemsetAsync(err, 0, sizeof(int32_t) * 8, s));
    CAV_CUDA(ctx, cudaMemsetAsync(bvh->nodes, 0, sizeof(BNode) * count, s));
    CAV_CUDA(ctx, cudaMemsetAsync(visited, 0, sizeof(uint32_t) * (n - 1), s));

    cudaEventRecord(bvh->ev[0], s);
    int32_t* bounds_ord = (int32_t*)(counters + 8);
    const int gb = div_up(n, kThreads);
    Bounds6 hb{};
    int use_dev = bounds ? 0 : 1;
    if (bounds) {
        for (int k = 0; k < 6; ++k) hb.v[k] = bounds[k];
        k_leaf_boxes<<<gb, kThreads, 0, s>>>(positions, indices, n, nv, leafbox, nullptr, err);
    } else {
        k_bounds_init<<<1, 32, 0, s>>>(bounds_ord);
        k_leaf_boxes<<<gb, kThreads, 0, s>>>(positions, indices, n, nv, leafbox, bounds_ord, err);
        k_bounds_decode<<<1, 32, 0, s>>>(bounds_ord, dbounds);
    }
    k_morton<<<gb, kThreads, 0, s>>>(leafbox, n, dbounds, hb, use_dev, bvh->codes_sorted, bvh->codes_unsorted, vals_a);
    cudaEventRecord(bvh->ev[1], s);

    // sort: 8 passes ping-ponging codes_sorted <-> keys_b, vals_a <-> vals_b; ends in A
    k_sort_hist<<<std::min(gb, ctx->num_sms * 8), kSortThreads, 0, s>>>(bvh->codes_sorted, n, 8, hist);
    CAV_CUDA(ctx, cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SortSmem)));
    uint64_t* kin = bvh->codes_sorted;
    uint64_t* kout = keys_b;
    uint32_t* vin = vals_a;
    uint32_t* vout = vals_b;
    for (int pass = 0; pass < 8; ++pass) {
        k_onesweep<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(kin, vin, kout, vout, n, 8 * pass, hist + 256 * pass,
                                                                  status + (size_t)pass * tiles * 256, counters + pass, err,
                                                                  ctx->sort_wait_ns, ctx->inject_sort_stall.load());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    cudaEventRecord(bvh->ev[2], s);

    k_radix_tree<<<div_up(n - 1, kThreads), kThreads, 0, s>>>(bvh->codes_sorted, (int32_t)n, bvh->nodes, err);
    cudaEventRecord(bvh->ev[3], s);
    k_refit<<<gb, kThreads, 0, s>>>(leafbox, vals_a, (int32_t)n, bvh->nodes, visited, err);
    cudaEventRecord(bvh->ev[4], s);
    CAV_CUDA(ctx, cudaMemcpyAsync(bvh->perm, vals_a, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    CAV_CUDA(ctx, cudaGetLastError());

    cav_status st = treelet_rounds(ctx, bvh->nodes, n, rounds, leaf_list, visited, counters + 14, s);
    if (st != CAV_OK) return st;
    cudaEventRecord(bvh->ev[5], s);

    // traversal layout
    int nblk = div_up(count, kScanTile);
    k_count_internal<<<nblk, kScanThreads, 0, s>>>(bvh->nodes, count, blk);
    k_scan_blocks<<<1, kScanThreads, 0, s>>>(blk, nblk);
    k_compact_index<<<nblk, kScanThreads, 0, s>>>(bvh->nodes, count, blk, compact);
    k_tri_layout<<<gb, kThreads, 0, s>>>(positions, nv, indices, mesh_ids, vals_a, n, bvh->tris, slot_of);
    k_tnode_layout<<<div_up(count, kThreads), kThreads, 0, s>>>(bvh->nodes, count, compact, slot_of, bvh->tnodes,
                                                                bvh->d_root_box);
    k_poison_tree<<<1, 32, 0, s>>>(err, bvh->tnodes, bvh->tris);
    cudaEventRecord(bvh->ev[6], s);
    CAV_CUDA(ctx, cudaGetLastError());
    k_merge_error<<<1, 32, 0, s>>>(err, ctx->d_error);
    CAV_CUDA(ctx, cudaFreeAsync(sbase, s));
    *out = bvh;
    return CAV_OK;
}

// ------------------------------------------------------------ many scenes, one launch
// A batch of scenes is built stage by stage with ONE launch per stage across all of them:
// leaf boxes and per-scene bounds, Morton codes (each scene against its own bounds), one
// stable sort of every code followed by one stable digit pass on the scene index (so each
// scene's codes end up contiguous and in the order a build of that scene alone gives),
// the radix trees of every scene, and the refits of every scene.  A thread finds its scene
// by binary search over the scenes' prefix offsets.  The treelet rounds and the traversal
// layout then run per scene.  Every scene gets its own cav_bvh, identical to cav_bvh_build's.
namespace {

struct BuildSeg {
    const float* pos;
    const int32_t* idx;
    int64_t n;
    int64_t nv;
    BNode* nodes;
    int32_t* perm;
    uint64_t* codes_sorted;
    uint64_t* codes_unsorted;
    float bounds[6];
    int use_dev;
};

__device__ inline int find_off(const int64_t* offs, int K, int64_t g) {
    int lo = 0, hi = K - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kThreads) k_leaf_boxes_batch(const BuildSeg* segs, const int64_t* leaf_offs, int K,
                                                               int64_t total, float* __restrict__ box,
                                                               int32_t* bounds_ord, int* err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g < total;
    int sg = -1;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool dev = false;
    if (valid) {
        sg = find_off(leaf_offs, K, g);
        const BuildSeg& S = segs[sg];
        const int64_t t = g - leaf_offs[sg];
        int32_t a, b, c;
        const bool ok = load_tri_idx(S.idx, t, S.nv, a, b, c, err);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float v0 = __ldg(S.pos + 3 * (int64_t)a + k), v1 = __ldg(S.pos + 3 * (int64_t)b + k),
                  v2 = __ldg(S.pos + 3 * (int64_t)c + k);
            lo[k] = fminf(v0, fminf(v1, v2));
            hi[k] = fmaxf(v0, fmaxf(v1, v2));
        }
        float* o = box + 6 * g;
        o[0] = lo[0]; o[1] = lo[1]; o[2] = lo[2];
        o[3] = hi[0]; o[4] = hi[1]; o[5] = hi[2];
        dev = S.use_dev != 0 && ok;
    }
    // bounds of the scenes without given bounds: a warp of one scene reduces first
    const unsigned same = __match_any_sync(0xffffffffu, valid && dev ? sg : -1);
    if (!(valid && dev)) return;
    if (same == 0xffffffffu) {
        int32_t v[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = __reduce_min_sync(0xffffffffu, f2ord(lo[k]));
            v[3 + k] = __reduce_max_sync(0xffffffffu, f2ord(hi[k]));
        }
        if ((threadIdx.x & 31) == 0) {
            for (int k = 0; k < 3; ++k) atomicMin(bounds_ord + 6 * sg + k, v[k]);
            for (int k = 0; k < 3; ++k) atomicMax(bounds_ord + 6 * sg + 3 + k, v[3 + k]);
        }
    } else {
        for (int k = 0; k < 3; ++k) atomicMin(bounds_ord + 6 * sg + k, f2ord(lo[k]));
        for (int k = 0; k < 3; ++k) atomicMax(bounds_ord + 6 * sg + 3 + k, f2ord(hi[k]));
    }
}

__global__ void k_bounds_batch(int32_t* bounds_ord, int K, int init, float* bounds) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 6 * K) return;
    if (init) bounds_ord[k] = (k % 6) < 3 ? INT32_MAX : INT32_MIN;
    else bounds[k] = ord2f(bounds_ord[k]);
}

__global__ void __launch_bounds__(kThreads) k_morton_batch(const float* __restrict__ box, const BuildSeg* segs,
                                                           const int64_t* leaf_offs, int K, int64_t total,
                                                           const float* dev_bounds, uint64_t* __restrict__ codes,
                                                           uint64_t* __restrict__ codes_copy, uint32_t* __restrict__ vals) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int sg = find_off(leaf_offs, K, g);
    const BuildSeg& S = segs[sg];
    const float* bb = S.use_dev ? dev_bounds + 6 * sg : S.bounds;
    f3 slo = mk(bb[0], bb[1], bb[2]), shi = mk(bb[3], bb[4], bb[5]);
    const float* b = box + 6 * g;
    f3 lo = mk(b[0], b[1], b[2]), hi = mk(b[3], b[4], b[5]);
    f3 centroid = ((lo + hi) * 0.5f - (slo + shi) * 0.5f) / (shi - slo);  // as k_morton
    uint64_t factor = (uint64_t)(1L << 21);
    uint64_t x = centroid.x * factor;
    uint64_t y = centroid.y * factor;
    uint64_t z = centroid.z * factor;
    uint64_t code = (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    codes[g] = code;
    codes_copy[g] = code;
    vals[g] = (uint32_t)g;
}

__global__ void k_scene_keys(const uint32_t* vals, const int64_t* leaf_offs, int K, int64_t total, uint64_t* key) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    key[i] = (uint64_t)find_off(leaf_offs, K, vals[i]);
}

// per scene: codes in triangle order and in sorted order, and the scene-local permutation
__global__ void k_scatter_batch(const uint64_t* codes_copy, const uint32_t* vals, const BuildSeg* segs,
                                const int64_t* leaf_offs, int K, int64_t total) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int sg = find_off(leaf_offs, K, g);
    const BuildSeg& S = segs[sg];
    const int64_t j = g - leaf_offs[sg];
    uint32_t t = vals[g];
    if ((int64_t)t < leaf_offs[sg] || (int64_t)t >= leaf_offs[sg + 1]) t = (uint32_t)leaf_offs[sg];  // failed sort
    S.codes_unsorted[j] = codes_copy[g];
    S.codes_sorted[j] = codes_copy[t];
    S.perm[j] = (int32_t)((int64_t)t - leaf_offs[sg]);
}

__global__ void __launch_bounds__(kThreads) k_radix_batch(const BuildSeg* segs, const int64_t* int_offs, int K,
                                                          int64_t total_internal, int* err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total_internal) return;
    const int sg = find_off(int_offs, K, g);
    const BuildSeg& S = segs[sg];
    radix_node(S.codes_sorted, (int32_t)S.n, S.nodes, (int32_t)(g - int_offs[sg]), err);
}

__global__ void __launch_bounds__(kThreads) k_refit_batch(const float* __restrict__ box, const uint32_t* vals,
                                                          const BuildSeg* segs, const int64_t* leaf_offs,
                                                          const int64_t* int_offs, int K, int64_t total,
                                                          uint32_t* visited, int* err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int sg = find_off(leaf_offs, K, g);
    const BuildSeg& S = segs[sg];
    const uint32_t t = vals[g];
    if ((int64_t)t < leaf_offs[sg] || (int64_t)t >= leaf_offs[sg + 1]) {  // outside its scene (a failed sort)
        atomicOr(err, kErrRefitLink);
        return;
    }
    refit_leaf(box, t, (int32_t)((int64_t)t - leaf_offs[sg]), (int32_t)S.n, S.nodes, visited + int_offs[sg],
               (int32_t)(g - leaf_offs[sg]), err);
}

}  // namespace

cav_status build_bvh_batch(cav_ctx* ctx, int K, const float* const* positions, const int64_t* num_vertices,
                           const int32_t* const* indices, const int32_t* const* mesh_ids, const int64_t* num_triangles,
                           const float* bounds, int rounds, cudaStream_t s, cav_bvh** out) {
    if (K < 1 || K > 65536 || !positions || !num_vertices || !indices || !num_triangles || !out || rounds < 0)
        return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_build_batch: invalid argument");
    std::vector<int64_t> leaf_offs(K + 1, 0), int_offs(K + 1, 0);
    int64_t nmax = 0;
    for (int k = 0; k < K; ++k) {
        const int64_t n = num_triangles[k];
        if (!positions[k] || !indices[k] || n < 2 || n >= (1ll << 30) || num_vertices[k] < 1)
            return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_build_batch: bad scene");
        leaf_offs[k + 1] = leaf_offs[k] + n;
        int_offs[k + 1] = int_offs[k] + n - 1;
        nmax = std::max(nmax, n);
    }
    const int64_t total = leaf_offs[K], total_int = int_offs[K];
    if (total >= (1ll << 32)) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "cav_bvh_build_batch: too many triangles");
    for (int k = 0; k < K; ++k) out[k] = nullptr;
    // one arena for every tree of the batch (one allocation, not K), stream-ordered; the trees
    // share it and the last one released frees it
    size_t arena_bytes = 0;
    for (int k = 0; k < K; ++k) arena_bytes += bvh_arena_bytes(num_triangles[k]) + 256;
    void* arena = nullptr;
    if (dev_alloc(ctx, &arena, arena_bytes, s, true) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "cav_bvh_build_batch: device allocation failed");
    }
    auto* shared = new SharedArena();
    shared->p = arena;
    shared->refs = K;
    std::vector<cav_bvh*> bv(K, nullptr);
    {
        unsigned char* p = (unsigned char*)arena;
        for (int k = 0; k < K; ++k) {
            p = (unsigned char*)(((uintptr_t)p + 255) & ~(uintptr_t)255);
            bv[k] = carve_bvh(ctx, num_triangles[k], p);
            bv[k]->shared = shared;
            p += bvh_arena_bytes(num_triangles[k]);
        }
    }
    auto fail = [&](cav_status st) {
        for (cav_bvh* b : bv) bvh_release(b, s, true);
        return st;
    };
    std::vector<BuildSeg> hs(K);
    for (int k = 0; k < K; ++k) {
        BuildSeg& g = hs[k];
        g.pos = positions[k];
        g.idx = indices[k];
        g.n = num_triangles[k];
        g.nv = num_vertices[k];
        g.nodes = bv[k]->nodes;
        g.perm = bv[k]->perm;
        g.codes_sorted = bv[k]->codes_sorted;
        g.codes_unsorted = bv[k]->codes_unsorted;
        g.use_dev = bounds ? 0 : 1;
        for (int c = 0; c < 6; ++c) g.bounds[c] = bounds ? bounds[6 * k + c] : 0.f;
    }
    const int tiles = div_up(total, kSortTile);
    const int passes2 = K <= 256 ? 1 : 2;
    const int64_t cmax = 2 * nmax - 1;
    size_t scratch = 0;
    auto acc = [&](size_t b) { scratch += b + 256; };
    acc(sizeof(BuildSeg) * K);
    acc(sizeof(int64_t) * (K + 1) * 2);
    acc(sizeof(float) * 6 * total);                 // leaf boxes
    acc(sizeof(uint64_t) * total * 3);              // codes, codes copy, ping-pong
    acc(sizeof(uint32_t) * total * 2);              // values ping-pong
    acc(sizeof(uint32_t) * 2 * 8 * 256);            // histograms (codes, scene keys)
    acc(sizeof(uint32_t) * (8 + passes2) * (size_t)tiles * 256);  // look-back status
    acc(sizeof(uint32_t) * 32);                     // tile counters
    acc(sizeof(int32_t) * 6 * K * 2);               // bounds (ordered ints, floats)
    acc(sizeof(int32_t) * 8);                       // error flag
    acc(sizeof(uint32_t) * std::max<int64_t>(total_int, 2 * total - K));  // visited (refit, then treelets)
    acc(sizeof(int32_t) * total);                   // leaf lists of all trees
    acc(sizeof(uint32_t) * (K + 2));                // leaf-list counters + treelet claim counters
    acc(sizeof(TreeletSeg) * K);                    // treelet table
    acc(sizeof(int32_t) * cmax);                    // compact index
    acc(sizeof(int32_t) * nmax);                    // slot_of
    acc(sizeof(uint32_t) * (div_up(cmax, kScanTile) + 1));
    void* sbase = nullptr;
    if (dev_alloc(ctx, &sbase, scratch, s, true) != cudaSuccess) {
        cudaGetLastError();
        return fail(set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "cav_bvh_build_batch: scratch allocation failed"));
    }
    unsigned char* q = (unsigned char*)sbase;
    BuildSeg* dsegs = carve<BuildSeg>(q, K);
    int64_t* d_leaf = carve<int64_t>(q, K + 1);
    int64_t* d_int = carve<int64_t>(q, K + 1);
    float* leafbox = carve<float>(q, 6 * total);
    uint64_t* codes = carve<uint64_t>(q, total);
    uint64_t* codes_copy = carve<uint64_t>(q, total);
    uint64_t* keys_b = carve<uint64_t>(q, total);
    uint32_t* vals_a = carve<uint32_t>(q, total);
    uint32_t* vals_b = carve<uint32_t>(q, total);
    uint32_t* hist = carve<uint32_t>(q, 2 * 8 * 256);
    uint32_t* status = carve<uint32_t>(q, (8 + passes2) * (size_t)tiles * 256);
    uint32_t* counters = carve<uint32_t>(q, 32);
    int32_t* bounds_ord = carve<int32_t>(q, 6 * K);
    float* dbounds = carve<float>(q, 6 * K);
    int32_t* err = carve<int32_t>(q, 8);
    uint32_t* visited = carve<uint32_t>(q, std::max<int64_t>(total_int, 2 * total - K));
    int32_t* leaf_list = carve<int32_t>(q, total);
    uint32_t* leaf_ctr = carve<uint32_t>(q, K + 2);
    TreeletSeg* tsegs = carve<TreeletSeg>(q, K);
    int32_t* compact = carve<int32_t>(q, cmax);
    int32_t* slot_of = carve<int32_t>(q, nmax);
    uint32_t* blk = carve<uint32_t>(q, div_up(cmax, kScanTile) + 1);
    // tables: stream-ordered copies from pageable host memory (staged before each call returns,
    // so the host vectors may go once the calls are made)
    CAV_CUDA(ctx, cudaMemcpyAsync(dsegs, hs.data(), sizeof(BuildSeg) * K, cudaMemcpyHostToDevice, s));
    CAV_CUDA(ctx, cudaMemcpyAsync(d_leaf, leaf_offs.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, s));
    CAV_CUDA(ctx, cudaMemcpyAsync(d_int, int_offs.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, s));
    std::vector<TreeletSeg> tsegs_host(K);
    for (int k = 0; k < K; ++k) tsegs_host[k] = TreeletSeg{bv[k]->nodes, num_triangles[k]};
    CAV_CUDA(ctx, cudaMemcpyAsync(tsegs, tsegs_host.data(), sizeof(TreeletSeg) * K, cudaMemcpyHostToDevice, s));
    CAV_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 2 * 8 * 256, s));
    CAV_CUDA(ctx, cudaMemsetAsync(status, 0, sizeof(uint32_t) * (8 + passes2) * (size_t)tiles * 256, s));
    CAV_CUDA(ctx, cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 32, s));
    CAV_CUDA(ctx, cudaMemsetAsync(err, 0, sizeof(int32_t) * 8, s));
    CAV_CUDA(ctx, cudaMemsetAsync(visited, 0, sizeof(uint32_t) * total_int, s));
    for (int k = 0; k < K; ++k) {
        CAV_CUDA(ctx, cudaMemsetAsync(bv[k]->nodes, 0, sizeof(BNode) * (2 * num_triangles[k] - 1), s));
        for (int e = 0; e < 7; ++e) cudaEventCreate(&bv[k]->ev[e]);
        bv[k]->timed = true;
        cudaEventRecord(bv[k]->ev[0], s);
    }
    const int gb = div_up(total, kThreads);
    if (!bounds) k_bounds_batch<<<div_up(6 * K, 256), 256, 0, s>>>(bounds_ord, K, 1, dbounds);
    k_leaf_boxes_batch<<<gb, kThreads, 0, s>>>(dsegs, d_leaf, K, total, leafbox, bounds_ord, err);
    if (!bounds) k_bounds_batch<<<div_up(6 * K, 256), 256, 0, s>>>(bounds_ord, K, 0, dbounds);
    k_morton_batch<<<gb, kThreads, 0, s>>>(leafbox, dsegs, d_leaf, K, total, dbounds, codes, codes_copy, vals_a);
    for (int k = 0; k < K; ++k) cudaEventRecord(bv[k]->ev[1], s);
    // sort by code (8 passes, stable), then by scene (1-2 passes, stable)
    CAV_CUDA(ctx, cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SortSmem)));
    k_sort_hist<<<std::min(gb, ctx->num_sms * 8), kSortThreads, 0, s>>>(codes, total, 8, hist);
    uint64_t* kin = codes;
    uint64_t* kout = keys_b;
    uint32_t* vin = vals_a;
    uint32_t* vout = vals_b;
    for (int pass = 0; pass < 8; ++pass) {
        k_onesweep<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(kin, vin, kout, vout, total, 8 * pass,
                                                                  hist + 256 * pass,
                                                                  status + (size_t)pass * tiles * 256, counters + pass,
                                                                  err, ctx->sort_wait_ns, ctx->inject_sort_stall.load());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    // kin/vin: codes in code order; now key by scene index
    k_scene_keys<<<gb, kThreads, 0, s>>>(vin, d_leaf, K, total, kin);
    k_sort_hist<<<std::min(gb, ctx->num_sms * 8), kSortThreads, 0, s>>>(kin, total, passes2, hist + 8 * 256);
    for (int pass = 0; pass < passes2; ++pass) {
        k_onesweep<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(kin, vin, kout, vout, total, 8 * pass,
                                                                  hist + 8 * 256 + 256 * pass,
                                                                  status + (size_t)(8 + pass) * tiles * 256,
                                                                  counters + 8 + pass, err, ctx->sort_wait_ns,
                                                                  ctx->inject_sort_stall.load());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    k_scatter_batch<<<gb, kThreads, 0, s>>>(codes_copy, vin, dsegs, d_leaf, K, total);
    for (int k = 0; k < K; ++k) cudaEventRecord(bv[k]->ev[2], s);
    k_radix_batch<<<div_up(total_int, kThreads), kThreads, 0, s>>>(dsegs, d_int, K, total_int, err);
    for (int k = 0; k < K; ++k) cudaEventRecord(bv[k]->ev[3], s);
    k_refit_batch<<<gb, kThreads, 0, s>>>(leafbox, vin, dsegs, d_leaf, d_int, K, total, visited, err);
    for (int k = 0; k < K; ++k) cudaEventRecord(bv[k]->ev[4], s);
    CAV_CUDA(ctx, cudaGetLastError());
    // treelet rounds of all scenes (two launches per round and group of scenes), then the
    // traversal layout per scene
    {
        cav_status st = treelet_rounds_batch(ctx, tsegs, tsegs_host.data(), d_leaf, leaf_offs.data(), K, rounds,
                                             leaf_list, leaf_ctr, visited, s);
        if (st != CAV_OK) {
            cudaFreeAsync(sbase, s);
            return fail(st);
        }
    }
    for (int k = 0; k < K; ++k) cudaEventRecord(bv[k]->ev[5], s);
    for (int k = 0; k < K; ++k) {
        cav_bvh* b = bv[k];
        const int64_t n = num_triangles[k], count = 2 * n - 1;
        const int nblk = div_up(count, kScanTile);
        k_count_internal<<<nblk, kScanThreads, 0, s>>>(b->nodes, count, blk);
        k_scan_blocks<<<1, kScanThreads, 0, s>>>(blk, nblk);
        k_compact_index<<<nblk, kScanThreads, 0, s>>>(b->nodes, count, blk, compact);
        k_tri_layout<<<div_up(n, kThreads), kThreads, 0, s>>>(positions[k], num_vertices[k], indices[k],
                                                             mesh_ids ? mesh_ids[k] : nullptr,
                                                             reinterpret_cast<const uint32_t*>(b->perm), n, b->tris,
                                                             slot_of);
        k_tnode_layout<<<div_up(count, kThreads), kThreads, 0, s>>>(b->nodes, count, compact, slot_of, b->tnodes,
                                                                    b->d_root_box);
        k_poison_tree<<<1, 32, 0, s>>>(err, b->tnodes, b->tris);
        cudaEventRecord(b->ev[6], s);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    k_merge_error<<<1, 32, 0, s>>>(err, ctx->d_error);
    CAV_CUDA(ctx, cudaFreeAsync(sbase, s));
    for (int k = 0; k < K; ++k) out[k] = bv[k];
    return CAV_OK;
}

size_t sort_status_words(int64_t n, int passes) { return (size_t)passes * div_up(n, kSortTile) * 256; }

cav_status sort_pairs(cav_ctx* ctx, uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, int64_t n,
                      int passes, uint32_t* hist, uint32_t* status, uint32_t* counters, int* err, cudaStream_t s) {
    if (n <= 0) return CAV_OK;
    if (passes <= 0 || passes > 8 || (passes & 1)) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "sort_pairs: passes");
    const int tiles = div_up(n, kSortTile);
    CAV_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, s));
    CAV_CUDA(ctx, cudaMemsetAsync(status, 0, sizeof(uint32_t) * sort_status_words(n, passes), s));
    CAV_CUDA(ctx, cudaMemsetAsync(counters, 0, sizeof(uint32_t) * passes, s));
    CAV_CUDA(ctx, cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SortSmem)));
    k_sort_hist<<<std::min(div_up(n, kThreads), ctx->num_sms * 8), kSortThreads, 0, s>>>(keys, n, passes, hist);
    uint64_t* kin = keys;
    uint64_t* kout = keys_tmp;
    uint32_t* vin = vals;
    uint32_t* vout = vals_tmp;
    for (int pass = 0; pass < passes; ++pass) {
        k_onesweep<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(kin, vin, kout, vout, n, 8 * pass, hist + 256 * pass,
                                                                  status + (size_t)pass * tiles * 256, counters + pass,
                                                                  err, ctx->sort_wait_ns, 0);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    return CAV_OK;
}

}  // namespace cav

// ------------------------------------------------------- allocation-free entry point
// Morton codes + stable sort (the first LBVH stages) for callers that cannot call
// cudaMalloc: for example a renderer embedded in a host application that hands out all
// device memory from its own pool fixed at start-up, or a per-frame loop that must not
// block on cudaMalloc (which may synchronise the device) or risk an allocation failure
// mid-frame.  Scratch lives in the file-scope array below, sized for at most
// CAV_NOALLOC_MAX_TRIANGLES triangles (about 4.8 MB; every GPU that loads this library
// keeps it until the process exits).  The sorted codes and the permutation are written
// straight into the caller's output buffers, which double as the sort's ping-pong side A.
namespace cav {
namespace {

constexpr int64_t kNoAllocMax = CAV_NOALLOC_MAX_TRIANGLES;
constexpr uint64_t kNoAllocSortWaitNs = 2000000000ull;  // the sort's look-back gives up after 2 s
constexpr int kNoAllocTiles = (int)((kNoAllocMax + kSortTile - 1) / kSortTile);
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffBox = 0;
constexpr size_t kOffKeys = kOffBox + align_up(sizeof(float) * 6 * kNoAllocMax);
constexpr size_t kOffVals = kOffKeys + align_up(sizeof(uint64_t) * kNoAllocMax);
constexpr size_t kOffHist = kOffVals + align_up(sizeof(uint32_t) * kNoAllocMax);
constexpr size_t kOffStatus = kOffHist + align_up(sizeof(uint32_t) * 8 * 256);
constexpr size_t kOffCounters = kOffStatus + align_up(sizeof(uint32_t) * 8 * (size_t)kNoAllocTiles * 256);
constexpr size_t kOffErr = kOffCounters + align_up(sizeof(uint32_t) * 16);
constexpr size_t kOffBounds = kOffErr + align_up(sizeof(int32_t) * 8);
constexpr size_t kNoAllocBytes = kOffBounds + align_up(sizeof(float) * 8);

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// The host-side name g_noalloc_scratch is only a stand-in for the symbol; its device
// address is looked up once per device (with that device current) and cached.
// The device's SM count, read at the same time, sizes the histogram grid.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};
int g_noalloc_sms[kMaxDevices] = {};

cav_status noalloc_scratch(unsigned char** out, int* num_sms) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        int sms = 0;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
            cudaGetLastError();
            return CAV_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        g_noalloc_sms[dev] = sms;
    }
    *out = g_noalloc_ptr[dev];
    *num_sms = g_noalloc_sms[dev];
    return CAV_OK;
}

}  // namespace
}  // namespace cav

extern "C" cav_status cav_morton_sort_noalloc(const float* positions, int64_t num_vertices, const int32_t* indices,
                                              int64_t num_triangles, const float* scene_bounds,
                                              uint64_t* sorted_codes, int32_t* sorted_prims, void* stream) {
    using namespace cav;
    const int64_t n = num_triangles;
    if (!positions || !indices || !sorted_codes || !sorted_prims || num_vertices < 1) return CAV_ERR_INVALID_ARGUMENT;
    if (n < 2 || n > kNoAllocMax) return CAV_ERR_INVALID_ARGUMENT;  // outside [2, CAV_NOALLOC_MAX_TRIANGLES]
    const int64_t nv = num_vertices;
    unsigned char* base = nullptr;
    int num_sms = 0;
    cav_status st = noalloc_scratch(&base, &num_sms);
    if (st != CAV_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    float* leafbox = reinterpret_cast<float*>(base + kOffBox);
    uint64_t* keys_b = reinterpret_cast<uint64_t*>(base + kOffKeys);
    uint32_t* vals_b = reinterpret_cast<uint32_t*>(base + kOffVals);
    uint32_t* hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kOffStatus);
    uint32_t* counters = reinterpret_cast<uint32_t*>(base + kOffCounters);
    int32_t* err = reinterpret_cast<int32_t*>(base + kOffErr);
    float* dbounds = reinterpret_cast<float*>(base + kOffBounds);
    const int tiles = div_up(n, kSortTile);
    uint64_t* keys_a = sorted_codes;
    uint32_t* vals_a = reinterpret_cast<uint32_t*>(sorted_prims);
    // the array keeps the previous call's contents: clear everything that must start at zero
    if (cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, sizeof(uint32_t) * 8 * (size_t)tiles * 256, s) != cudaSuccess ||
        cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 16, s) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int32_t) * 8, s) != cudaSuccess) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    const int gb = div_up(n, kThreads);
    Bounds6 hb{};
    int use_dev = scene_bounds ? 0 : 1;
    int32_t* bounds_ord = reinterpret_cast<int32_t*>(counters + 8);
    if (scene_bounds) {
        for (int k = 0; k < 6; ++k) hb.v[k] = scene_bounds[k];
        k_leaf_boxes<<<gb, kThreads, 0, s>>>(positions, indices, n, nv, leafbox, nullptr, err);
    } else {
        k_bounds_init<<<1, 32, 0, s>>>(bounds_ord);
        k_leaf_boxes<<<gb, kThreads, 0, s>>>(positions, indices, n, nv, leafbox, bounds_ord, err);
        k_bounds_decode<<<1, 32, 0, s>>>(bounds_ord, dbounds);
    }
    // keys_b receives the unsorted copy; the first sort pass overwrites it
    k_morton<<<gb, kThreads, 0, s>>>(leafbox, n, dbounds, hb, use_dev, keys_a, keys_b, vals_a);
    k_sort_hist<<<std::min(gb, num_sms * 8), kSortThreads, 0, s>>>(keys_a, n, 8, hist);
    if (cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SortSmem)) !=
        cudaSuccess) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    uint64_t* kin = keys_a;
    uint64_t* kout = keys_b;
    uint32_t* vin = vals_a;
    uint32_t* vout = vals_b;
    for (int pass = 0; pass < 8; ++pass) {
        k_onesweep<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(kin, vin, kout, vout, n, 8 * pass, hist + 256 * pass,
                                                                  status + (size_t)pass * tiles * 256, counters + pass,
                                                                  err, kNoAllocSortWaitNs, 0);
        uint64_t* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    // 8 passes: the result is back in side A, the caller's buffers
    if (cudaGetLastError() != cudaSuccess) return CAV_ERR_CUDA;
    int32_t herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return CAV_ERR_CUDA;
    }
    if (herr == 0) return CAV_OK;
    if (herr & kErrLookback) return CAV_ERR_TIMEOUT;
    if (herr & kErrBadIndex) return CAV_ERR_INVALID_ARGUMENT;
    return CAV_ERR_CUDA;  // a sort invariant broke (kErrSortScatter)
}

