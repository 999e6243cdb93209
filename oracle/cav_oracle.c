/*
 * Cavalry BVH oracle — TEST INFRASTRUCTURE, not part of the product.
 *
 * A CPU restatement (plain C, scalar, one thread unless stated) of the reference's
 * LBVH build, treelet restructuring and ray traversal.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it, always as the checker or the timed CPU
 * baseline, never as the thing shipped.
 *
 * Reference files followed (paths inside AmesingFlank/Cavalry):
 *   Core/Triangle.h:242-268      leaf boxes                  -> orc_leaf_boxes
 *   Core/Scene.cu:131-135        host scene-bounds fold      -> orc_scene_bounds
 *   BVH/BVH.cu:46-56             fillLeafBoundingBoxes       -> orc_leaf_boxes (+area/cost)
 *   BVH/BVH.cu:59-92             shiftMorton/fillLeafMortonCodes -> orc_morton
 *   BVH/BVH.cu:335               thrust::stable_sort_by_key  -> orc_sort (LSD radix, stable)
 *   BVH/BVH.cu:96-215            sign/commonPrefixLength/buildRadixTree -> radix_tree
 *   BVH/BVH.cu:217-259           computeBounds               -> refit
 *   BVH/BVH.cu:261-302           copyLeafNode/mergeNodesArray -> merge
 *   BVH/Optimization.cu:20-462   optimizationSchedule/optimizeTreelet -> treelet
 *   BVH/Optimization.cu:467-525  optimizeBVHImpl/optimizeBVH -> treelet_round
 *   BVH/BVH.cu:304-315           copyToBVH                   -> (final array is the same records)
 *   BVH/SAH.h:4-21               leafCost/internalCost (FP64 literals)
 *   Core/BoundingBox.h:56-96     AABB::intersect/computeSurfaceArea/unionBoxes
 *   Utils/MathsCommons.h:93-100  vmin/vmax signed-int min/max on float bits
 *   Core/Triangle.h:7-57         rayTriangleIntersection (Moller-Trumbore)
 *   BVH/BVH.h:23-189             BVH::intersect / BVH::testVisibility
 *
 * Numerics.  The reference is compiled with -use_fast_math: denormals flush to zero,
 * and multiply-adds are contracted into FMAs.  This file is compiled with
 * -ffp-contract=off and writes the reference's contractions out as explicit fmaf/fma
 * calls; every entry point sets FTZ/DAZ in MXCSR for its duration.  The reference's
 * divisions and reciprocals compile to approximate GPU instructions that this file
 * does not imitate: it divides with IEEE division.  Morton codes may therefore differ
 * from the GPU's by one quantisation step on an axis where the quotient sits within a
 * few ulp of a cell boundary, and hit distances by a few ulp; the tests state those
 * tolerances.  All integer stages (sort, radix tree, treelet choice given identical
 * costs) are exact.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#include <pmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    float bmin[3];
    float bmax[3];
    int32_t begin, end, left, right, parent, is_leaf;
    float area, cost;
} ONode; /* 56 bytes; same field order as the harness dump of BVHRestructureNode */

/* ---------------------------------------------------------------- fp env */
static unsigned fp_enter(void) {
    unsigned old = _mm_getcsr();
    _mm_setcsr(old | 0x8040); /* FTZ (bit 15) | DAZ (bit 6) */
    return old;
}
static void fp_leave(unsigned old) { _mm_setcsr(old); }

/* ------------------------------------------------------- small fp helpers */
/* AABB::computeSurfaceArea, Core/BoundingBox.h:77-80:
 *   2.f*(ex*ey + ey*ez + ex*ez), contracted as fma(ex, ez, fma(ex, ey, ey*ez)). */
static float surface_area(const float* bmin, const float* bmax) {
    float ex = bmax[0] - bmin[0];
    float ey = bmax[1] - bmin[1];
    float ez = bmax[2] - bmin[2];
    float s = fmaf(ex, ez, fmaf(ex, ey, ey * ez));
    return 2.0f * s;
}
/* SAH.h:10-12: area * 1.0 * n in double, returned as float. */
static float leaf_cost(float area, int n) { return (float)((double)area * 1.0 * (double)n); }
/* SAH.h:15-17: area * 1.2 + l + r in double (first add contracted), returned as float. */
static float internal_cost3(float area, float l, float r) {
    return (float)(fma((double)area, 1.2, (double)l) + (double)r);
}
/* SAH.h:20-22 */
static float internal_cost2(float area, float c) { return (float)fma((double)area, 1.2, (double)c); }

static void box_union(const float* amin, const float* amax, const float* bmin, const float* bmax,
                      float* omin, float* omax) {
    for (int k = 0; k < 3; ++k) {
        omin[k] = fminf(amin[k], bmin[k]);
        omax[k] = fmaxf(amax[k], bmax[k]);
    }
}

/* ------------------------------------------------------------ leaf boxes */
void orc_leaf_boxes(const float* pos, const int32_t* idx, int64_t n, float* box) {
    unsigned f = fp_enter();
    for (int64_t i = 0; i < n; ++i) {
        const float* v0 = pos + 3 * (int64_t)idx[3 * i + 0];
        const float* v1 = pos + 3 * (int64_t)idx[3 * i + 1];
        const float* v2 = pos + 3 * (int64_t)idx[3 * i + 2];
        for (int k = 0; k < 3; ++k) {
            box[6 * i + k] = fminf(v0[k], fminf(v1[k], v2[k]));
            box[6 * i + 3 + k] = fmaxf(v0[k], fmaxf(v1[k], v2[k]));
        }
    }
    fp_leave(f);
}

void orc_scene_bounds(const float* box, int64_t n, float* out) {
    for (int k = 0; k < 6; ++k) out[k] = box[k];
    for (int64_t i = 1; i < n; ++i) box_union(out, out + 3, box + 6 * i, box + 6 * i + 3, out, out + 3);
}

/* ---------------------------------------------------------------- Morton */
/* shiftMorton, BVH/BVH.cu:59-76.  Clamp: `1 << MORTEN_BITS_PER_DIMENSION - 1` parses as
 * 1 << 20.  The five mask steps spread bit k of the 21-bit input to bit 3k. */
static uint64_t spread3(uint64_t x) {
    if (x >= (1ull << 21)) x = 1ull << 20;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

/* float -> uint64 as the GPU's cvt.rzi.u64.f32 does: truncation, negatives and NaN
 * saturate to 0, values >= 2^64 to UINT64_MAX. */
static uint64_t f2u64_sat(float v) {
    if (!(v > 0.0f)) return 0;
    if (v >= 18446744073709551616.0f) return UINT64_MAX;
    return (uint64_t)v;
}

void orc_morton(const float* box, int64_t n, const float* bounds, uint64_t* codes) {
    unsigned f = fp_enter();
    float sc[3], se[3];
    for (int k = 0; k < 3; ++k) {
        sc[k] = (bounds[k] + bounds[3 + k]) * 0.5f;
        se[k] = bounds[3 + k] - bounds[k];
    }
    const float factor = 2097152.0f; /* (float)(1L << 21) */
    for (int64_t i = 0; i < n; ++i) {
        uint64_t q[3];
        for (int k = 0; k < 3; ++k) {
            float c = (box[6 * i + k] + box[6 * i + 3 + k]) * 0.5f;
            float r = (c - sc[k]) / se[k];
            q[k] = f2u64_sat(r * factor);
            /* Zero scene extent on an axis: every centroid equals the scene centre and the
             * quotient is 0/0.  IEEE gives NaN (-> cell 0); the reference's fast-math GPU
             * division puts every such centroid in the clamped top cell (1 << 20), as its
             * own outputs show (tests/golden/flat2k.npz).  The oracle follows the reference. */
            if (se[k] == 0.0f) q[k] = UINT64_MAX;
        }
        codes[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    }
    fp_leave(f);
}

/* ------------------------------------------------------------------ sort */
/* Stable ascending sort of 64-bit keys carrying the original index, as
 * thrust::stable_sort_by_key (BVH/BVH.cu:335) leaves it.  LSD radix, 16-bit digits. */
void orc_sort(const uint64_t* codes, int64_t n, uint64_t* sorted, int32_t* perm) {
    uint64_t* ka = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t* kb = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int32_t* va = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* vb = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * 65536);
    for (int64_t i = 0; i < n; ++i) {
        ka[i] = codes[i];
        va[i] = (int32_t)i;
    }
    for (int pass = 0; pass < 4; ++pass) {
        int sh = 16 * pass;
        memset(cnt, 0, sizeof(int64_t) * 65536);
        for (int64_t i = 0; i < n; ++i) cnt[(ka[i] >> sh) & 0xffff]++;
        int64_t s = 0;
        for (int d = 0; d < 65536; ++d) {
            int64_t c = cnt[d];
            cnt[d] = s;
            s += c;
        }
        for (int64_t i = 0; i < n; ++i) {
            int64_t p = cnt[(ka[i] >> sh) & 0xffff]++;
            kb[p] = ka[i];
            vb[p] = va[i];
        }
        uint64_t* tk = ka; ka = kb; kb = tk;
        int32_t* tv = va; va = vb; vb = tv;
    }
    memcpy(sorted, ka, sizeof(uint64_t) * (size_t)n);
    memcpy(perm, va, sizeof(int32_t) * (size_t)n);
    free(ka); free(kb); free(va); free(vb); free(cnt);
}

/* ------------------------------------------------------------ radix tree */
/* commonPrefixLength, BVH/BVH.cu:101-120: differing codes -> number of equal leading
 * bits among the 63 code bits; equal codes -> 63 + equal leading bits of the 32-bit
 * indices; 95 when i == j. */
static int cpl(const uint64_t* m, uint32_t i, uint32_t j) {
    uint64_t a = m[i], b = m[j];
    if (a != b) {
        for (int bit = 62; bit >= 0; --bit)
            if (((a >> bit) & 1) != ((b >> bit) & 1)) return 62 - bit;
    }
    for (int bit = 31; bit >= 0; --bit)
        if (((i >> bit) & 1) != ((j >> bit) & 1)) return (31 - bit) + 63;
    return 95;
}

typedef struct {
    float bmin[3], bmax[3];
    int32_t left, right, parent;
    uint32_t visited;
    uint8_t lleaf, rleaf;
    float area, cost;
} OInternal;

typedef struct {
    float bmin[3], bmax[3];
    int32_t begin, end, parent;
    float area, cost;
} OLeaf;

/* buildRadixTree, BVH/BVH.cu:122-215, one iteration per internal node i. */
static void radix_tree(int32_t N, const uint64_t* m, OLeaf* leaves, OInternal* in) {
    for (int32_t i = 0; i < N - 1; ++i) {
        int d = 1;
        if (i > 0) d = (cpl(m, i, i + 1) - cpl(m, i, i - 1)) >= 0 ? 1 : -1;
        int minCPL = 0;
        if (i > 0) minCPL = cpl(m, i, (uint32_t)(i - d));
        /* unsigned arithmetic of :137-141; the wrapped value can never land in [0, N) */
        uint32_t maxLength = 2;
        for (;;) {
            int64_t jj = (int64_t)i + (int64_t)maxLength * d;
            if (!(jj >= 0 && jj < N)) break;
            if (!(cpl(m, i, (uint32_t)jj) > minCPL)) break;
            maxLength *= 2;
        }
        uint32_t length = 0;
        for (int power = 1;; ++power) {
            uint32_t t = maxLength >> power;
            if (t == 0) break;
            int32_t j = (int32_t)((uint32_t)i + (length + t) * (uint32_t)d);
            if (j >= 0 && j < N && cpl(m, i, j) > minCPL) length += t;
        }
        int32_t j = (int32_t)((uint32_t)i + length * (uint32_t)d);
        if (i == 0) j = N - 1;
        int prefix = cpl(m, i, j);
        uint32_t dist = 0;
        for (int power = 1;; ++power) {
            /* :169  ceil((float)length / (float)(1<<power)); exact division by 2^p */
            uint32_t t = (uint32_t)ceilf((float)length / (float)(1 << power));
            int32_t jj = (int32_t)((uint32_t)i + (dist + t) * (uint32_t)d);
            if (jj >= 0 && jj < N && cpl(m, i, jj) > prefix) dist += t;
            if (t <= 1) break;
        }
        int32_t split = (int32_t)((uint32_t)i + dist * (uint32_t)d) + (d < 0 ? d : 0);
        int32_t lc = split, rc = split + 1;
        in[i].left = lc;
        in[i].right = rc;
        int32_t mn = i < j ? i : j, mx = i > j ? i : j;
        in[i].lleaf = (mn == lc);
        in[i].rleaf = (mx == rc) || (rc == N - 1);
        if (in[i].lleaf) leaves[lc].parent = i; else in[lc].parent = i;
        if (in[i].rleaf) leaves[rc].parent = i; else in[rc].parent = i;
        in[i].visited = 0;
    }
}

/* computeBounds, BVH/BVH.cu:217-259: the second arrival at a node unions the child
 * boxes.  Values do not depend on arrival order, so leaves are walked in index order. */
static void refit(int32_t N, OLeaf* leaves, OInternal* in) {
    for (int32_t i = 0; i < N; ++i) {
        int32_t curr = leaves[i].parent;
        for (;;) {
            uint32_t old = in[curr].visited;
            in[curr].visited = old >= 2 ? 0 : old + 1; /* atomicInc(.., 2) */
            if (old == 0) break;
            OInternal* nd = &in[curr];
            const float *lmin, *lmax, *rmin, *rmax;
            float cl, cr;
            if (nd->lleaf) { lmin = leaves[nd->left].bmin; lmax = leaves[nd->left].bmax; cl = leaves[nd->left].cost; }
            else { lmin = in[nd->left].bmin; lmax = in[nd->left].bmax; cl = in[nd->left].cost; }
            if (nd->rleaf) { rmin = leaves[nd->right].bmin; rmax = leaves[nd->right].bmax; cr = leaves[nd->right].cost; }
            else { rmin = in[nd->right].bmin; rmax = in[nd->right].bmax; cr = in[nd->right].cost; }
            box_union(lmin, lmax, rmin, rmax, nd->bmin, nd->bmax);
            nd->area = surface_area(nd->bmin, nd->bmax);
            nd->cost = internal_cost3(nd->area, cl, cr);
            if (curr == 0) break;
            curr = nd->parent;
        }
    }
}

/* mergeNodesArray, BVH/BVH.cu:273-302: internals at [0, N-2], leaf i at N-1+i.
 * Fields the reference never writes stay 0 (GpuArray zero-fills, Utils/Array.h:102-108). */
static void merge(int32_t N, const OLeaf* leaves, const OInternal* in, ONode* nodes) {
    memset(nodes, 0, sizeof(ONode) * (size_t)(2 * N - 1));
    for (int32_t i = 0; i < N - 1; ++i) {
        ONode* n = &nodes[i];
        n->is_leaf = 0;
        n->parent = in[i].parent;
        memcpy(n->bmin, in[i].bmin, 12);
        memcpy(n->bmax, in[i].bmax, 12);
        n->area = in[i].area;
        n->cost = in[i].cost;
        int32_t sides[2] = {in[i].left, in[i].right};
        uint8_t isl[2] = {in[i].lleaf, in[i].rleaf};
        for (int s = 0; s < 2; ++s) {
            if (isl[s]) {
                int32_t li = N - 1 + sides[s];
                if (s == 0) n->left = li; else n->right = li;
                const OLeaf* L = &leaves[sides[s]];
                ONode* d = &nodes[li];
                memcpy(d->bmin, L->bmin, 12);
                memcpy(d->bmax, L->bmax, 12);
                d->parent = L->parent;
                d->is_leaf = 1;
                d->begin = L->begin;
                d->end = L->end;
                d->area = L->area;
                d->cost = L->cost;
            } else {
                if (s == 0) n->left = sides[s]; else n->right = sides[s];
            }
        }
    }
}

/* --------------------------------------------------------------- treelet */
/* optimizationSchedule, BVH/Optimization.cu:20-47 (32 lanes x 5 rounds). */
static const uint8_t kSchedule[160] = {
    0x03, 0x06, 0x05, 0x09, 0x0a, 0x0c, 0x11, 0x12, 0x14, 0x18, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0x07, 0x0b, 0x0d, 0x0e, 0x13, 0x15, 0x16, 0x19, 0x1a, 0x1c, 0x21, 0x22, 0x24, 0x28, 0x30, 0x41, 0x42, 0x44, 0x48, 0x50, 0x60, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0x23, 0x25, 0x26, 0x29, 0x2a, 0x2c, 0x31, 0x32, 0x34, 0x38, 0x43, 0x45, 0x46, 0x49, 0x4a, 0x4c, 0x51, 0x52, 0x54, 0x58, 0x61, 0x62, 0x64, 0x68, 0x70, 0x0f, 0x17, 0x1e, 0, 0, 0, 0,
    0x47, 0x1b, 0x2b, 0x4b, 0x33, 0x53, 0x63, 0x1d, 0x2d, 0x4d, 0x35, 0x55, 0x65, 0x39, 0x59, 0x69, 0x71, 0x27, 0x2e, 0x4e, 0x36, 0x56, 0x66, 0x3a, 0x5a, 0x6a, 0x72, 0x3c, 0x5c, 0x6c, 0x74, 0x78,
    0x1f, 0x2f, 0x4f, 0x37, 0x57, 0x67, 0x3b, 0x5b, 0x6b, 0x73, 0x3d, 0x5d, 0x6d, 0x75, 0x79, 0x3e, 0x5e, 0x6e, 0x76, 0x7a, 0x7c, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
};

/* Lane-order min reduction of Optimization.cu:252-261 / :311-319, with shfl snapshot
 * semantics: at step d lane l takes lane min(l+d,31)'s pair if its own cost is -1 or
 * the other cost is strictly smaller.  Returns lane 0's pair. */
static void warp_min_reduce(float* cost, int* part) {
    for (int d = 16; d >= 1; d >>= 1) {
        float oc[32];
        int op[32];
        for (int l = 0; l < 32; ++l) {
            int o = l + d < 31 ? l + d : 31;
            oc[l] = cost[o];
            op[l] = part[o];
        }
        for (int l = 0; l < 32; ++l) {
            if (cost[l] == -1.0f || oc[l] < cost[l]) {
                cost[l] = oc[l];
                part[l] = op[l];
            }
        }
    }
}

static int is_pow2(int n) { return (n & (n - 1)) == 0; }

/* optimizeTreelet, BVH/Optimization.cu:49-462, one warp simulated lane by lane. */
static void treelet(ONode* nodes, int32_t root) {
    int32_t my_node[32];
    int expanded[32];
    for (int l = 0; l < 32; ++l) { my_node[l] = -1; expanded[l] = 0; }
    my_node[0] = root;

    /* formation, :59-107 */
    int size = 1;
    while (size < 13) {
        int max_lane = 0;
        float max_area = -1.0f;
        for (int i = 0; i < size; ++i) {
            float a = nodes[my_node[i]].area;
            if (nodes[my_node[i]].is_leaf || expanded[i]) a = -1.0f;
            if (a > max_area) { max_area = a; max_lane = i; }
        }
        if (expanded[max_lane] || nodes[my_node[max_lane]].is_leaf) return; /* fewer than 7 leaves */
        expanded[max_lane] = 1;
        int32_t x = my_node[max_lane];
        my_node[size] = nodes[x].left;
        my_node[size + 1] = nodes[x].right;
        size += 2;
    }
    int32_t leaves[7];
    int nl = 0;
    for (int i = 0; i < 13; ++i)
        if (!expanded[i]) leaves[nl++] = my_node[i];

    /* subset areas, :126-163 */
    float area[128], opt_cost[128];
    int opt_part[128];
    for (int s = 0; s < 128; ++s) {
        int any = 0;
        float bmin[3], bmax[3];
        for (int b = 0; b < 7; ++b) {
            if (!((s >> b) & 1)) continue;
            const ONode* L = &nodes[leaves[b]];
            if (!any) { memcpy(bmin, L->bmin, 12); memcpy(bmax, L->bmax, 12); any = 1; }
            else box_union(bmin, bmax, L->bmin, L->bmax, bmin, bmax);
        }
        area[s] = any ? surface_area(bmin, bmax) : 0.0f;
        opt_cost[s] = -1.0f;
        opt_part[s] = 0;
    }
    for (int i = 0; i < 7; ++i) opt_cost[1 << i] = nodes[leaves[i]].cost;

    /* scheduled DP for subsets of 2..5 leaves, :180-216 (lanes of a round are
     * independent; results are written after all lanes computed, as in lockstep) */
    for (int round = 0; round < 5; ++round) {
        float rc[32];
        int rp[32];
        for (int lane = 0; lane < 32; ++lane) {
            int s = kSchedule[round * 32 + lane];
            if (!s) continue;
            float best = -1.0f;
            int bestp = 0;
            int cleared = (s - 1) & s;
            int p = (0 - cleared) & s;
            do {
                float tc = opt_cost[p] + opt_cost[s ^ p];
                if (best == -1.0f || tc < best) { bestp = p; best = tc; }
                p = (p - cleared) & s;
            } while (p != 0);
            rc[lane] = internal_cost2(area[s], best);
            rp[lane] = bestp;
        }
        for (int lane = 0; lane < 32; ++lane) {
            int s = kSchedule[round * 32 + lane];
            if (!s) continue;
            opt_cost[s] = rc[lane];
            opt_part[s] = rp[lane];
        }
    }

    /* 6-leaf subsets, :224-266.  `consequtiveBits(5-emptyBit)` with emptyBit = 6 is a
     * shift by -1; on the GPU that shift yields 0, giving an all-ones mask. */
    for (int e = 0; e < 7; ++e) {
        int s = 0x7f ^ (1 << e);
        float tc[32];
        int pp[32];
        for (int lane = 0; lane < 32; ++lane) {
            int lo = lane & ((1 << e) - 1);
            int himask = (5 - e >= 0) ? ((1 << (5 - e)) - 1) : -1;
            int p = (lo | ((lane << 1) & (int)((unsigned)himask << (e + 1)))) & 0xff;
            p = (int)(signed char)p;
            tc[lane] = -1.0f;
            pp[lane] = p;
            if (p != 0) tc[lane] = opt_cost[p] + opt_cost[s ^ p];
        }
        warp_min_reduce(tc, pp);
        opt_cost[s] = internal_cost2(area[s], tc[0]);
        opt_part[s] = pp[0];
    }

    /* all 7 leaves, :271-324 */
    {
        int s = 0x7f;
        float tc[32];
        int pp[32];
        for (int lane = 0; lane < 32; ++lane) {
            int p = lane;
            float t = -1.0f;
            if (p != 0) t = opt_cost[p] + opt_cost[s ^ p];
            int op = lane | 32;
            float ot = opt_cost[op] + opt_cost[s ^ op];
            if (t == -1.0f || ot < t) { t = ot; p = op; }
            tc[lane] = t;
            pp[lane] = p;
        }
        warp_min_reduce(tc, pp);
        opt_cost[s] = internal_cost2(area[s], tc[0]);
        opt_part[s] = pp[0];
    }

    /* reconstruction, :330-394: lane i keeps node my_node[i] and takes a new role */
    int my_subset[32], exp_r[32], my_parent[32];
    int32_t new_left[32], new_right[32]; /* indexed by lane (node my_node[lane]) */
    for (int l = 0; l < 32; ++l) { my_subset[l] = -1; exp_r[l] = 0; my_parent[l] = -1; new_left[l] = -1; new_right[l] = -1; }
    my_subset[0] = 0x7f;
    my_parent[0] = nodes[my_node[0]].parent;
    int rsize = 1;
    while (rsize < 13) {
        int sel = -1, sel_lane = -1;
        for (int i = 0; i < rsize; ++i) {
            int prop = (!exp_r[i] && !is_pow2(my_subset[i])) ? my_subset[i] : -1;
            if (prop != -1 && sel == -1) { sel = prop; sel_lane = i; }
        }
        if (sel_lane < 0) return; /* cannot happen for a 7-leaf treelet */
        exp_r[sel_lane] = 1;
        int32_t parent_node = my_node[sel_lane];
        my_parent[rsize] = parent_node;
        my_subset[rsize] = opt_part[sel];
        new_left[sel_lane] = my_node[rsize];
        my_parent[rsize + 1] = parent_node;
        my_subset[rsize + 1] = sel ^ opt_part[sel];
        new_right[sel_lane] = my_node[rsize + 1];
        rsize += 2;
    }

    /* write-back, :400-461.  Reads of the old treelet leaves happen before any
     * lane overwrites a node (lockstep order of the reference). */
    int nleaf[13];
    float nbmin[13][3], nbmax[13][3];
    int32_t nbegin[13], nend[13];
    for (int l = 0; l < 13; ++l) {
        int32_t me = my_node[l];
        nodes[me].parent = my_parent[l];
        if (!exp_r[l]) {
            int leaf_id = 0;
            int t = my_subset[l];
            while ((t & 1) == 0) { ++leaf_id; t >>= 1; }
            const ONode* o = &nodes[leaves[leaf_id]];
            nleaf[l] = o->is_leaf;
            nbegin[l] = o->begin;
            nend[l] = o->end;
            memcpy(nbmin[l], o->bmin, 12);
            memcpy(nbmax[l], o->bmax, 12);
            new_left[l] = o->left;
            new_right[l] = o->right;
            if (!o->is_leaf) {
                nodes[o->left].parent = me;
                nodes[o->right].parent = me;
            }
        } else {
            nleaf[l] = 0;
            nbegin[l] = 0;
            nend[l] = 0;
        }
    }
    for (int l = 0; l < 13; ++l) {
        ONode* n = &nodes[my_node[l]];
        n->left = new_left[l];
        n->right = new_right[l];
        n->is_leaf = nleaf[l];
        if (!exp_r[l]) {
            n->begin = nbegin[l];
            n->end = nend[l];
            memcpy(n->bmin, nbmin[l], 12);
            memcpy(n->bmax, nbmax[l], 12);
            n->area = surface_area(n->bmin, n->bmax);
        } else {
            /* the reference stores an uninitialised box/prim range here and then
             * overwrites box/area in the refresh loop; prim range stays unspecified */
            n->begin = -1;
            n->end = -1;
        }
    }
    /* refresh loop :445-460 converges to a bottom-up recompute; children always sit
     * at higher lanes than their parent, so descending lane order is bottom-up. */
    for (int l = 12; l >= 0; --l) {
        ONode* n = &nodes[my_node[l]];
        if (exp_r[l]) {
            const ONode* a = &nodes[n->left];
            const ONode* b = &nodes[n->right];
            box_union(a->bmin, a->bmax, b->bmin, b->bmax, n->bmin, n->bmax);
            n->area = surface_area(n->bmin, n->bmax);
        }
        if (n->is_leaf) n->cost = leaf_cost(n->area, n->end - n->begin + 1);
        else n->cost = internal_cost3(n->area, nodes[n->left].cost, nodes[n->right].cost);
    }
}

/* optimizeBVHImpl, BVH/Optimization.cu:467-507: warps start at the nodes that are
 * leaves when the round begins and walk up; the second arrival optimises the parent. */
static void treelet_round(ONode* nodes, int32_t count) {
    uint32_t* visited = (uint32_t*)calloc((size_t)count, sizeof(uint32_t));
    int32_t* starts = (int32_t*)malloc(sizeof(int32_t) * (size_t)count);
    int32_t ns = 0;
    for (int32_t i = 0; i < count; ++i)
        if (nodes[i].is_leaf) starts[ns++] = i;
    for (int32_t k = 0; k < ns; ++k) {
        int32_t curr = starts[k];
        for (;;) {
            if (!nodes[curr].is_leaf) treelet(nodes, curr);
            if (curr == 0) break;
            int32_t parent = nodes[curr].parent;
            uint32_t old = visited[parent];
            visited[parent] = old >= 2 ? 0 : old + 1;
            if (old != 1) break;
            curr = parent;
        }
    }
    free(visited);
    free(starts);
}

/* ------------------------------------------------------------- build API */
/* Full build.  codes_in (optional): unsorted Morton codes to use instead of computing
 * them (lets the integer stages be checked exactly against GPU-computed codes).
 * Outputs (optional): codes_out (unsorted), sorted_codes, perm, merged (2N-1),
 * final (2N-1), bounds_out (6). */
int orc_build(const float* pos, const int32_t* idx, int64_t n, const float* bounds_in, const uint64_t* codes_in,
              int rounds, uint64_t* codes_out, uint64_t* sorted_out, int32_t* perm_out, ONode* merged,
              ONode* final_nodes, float* bounds_out) {
    if (n < 2 || n > 0x3fffffff) return -1;
    unsigned f = fp_enter();
    int32_t N = (int32_t)n;
    float* box = (float*)malloc(sizeof(float) * 6 * (size_t)N);
    orc_leaf_boxes(pos, idx, N, box);
    float bounds[6];
    if (bounds_in) memcpy(bounds, bounds_in, 24);
    else orc_scene_bounds(box, N, bounds);
    if (bounds_out) memcpy(bounds_out, bounds, 24);
    uint64_t* codes = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)N);
    if (codes_in) memcpy(codes, codes_in, sizeof(uint64_t) * (size_t)N);
    else orc_morton(box, N, bounds, codes);
    if (codes_out) memcpy(codes_out, codes, sizeof(uint64_t) * (size_t)N);
    uint64_t* sorted = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)N);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    orc_sort(codes, N, sorted, perm);
    if (sorted_out) memcpy(sorted_out, sorted, sizeof(uint64_t) * (size_t)N);
    if (perm_out) memcpy(perm_out, perm, sizeof(int32_t) * (size_t)N);

    OLeaf* leaves = (OLeaf*)calloc((size_t)N, sizeof(OLeaf));
    for (int32_t i = 0; i < N; ++i) {
        int32_t t = perm[i];
        memcpy(leaves[i].bmin, box + 6 * (size_t)t, 12);
        memcpy(leaves[i].bmax, box + 6 * (size_t)t + 3, 12);
        leaves[i].begin = t;
        leaves[i].end = t;
        leaves[i].area = surface_area(leaves[i].bmin, leaves[i].bmax);
        leaves[i].cost = leaf_cost(leaves[i].area, 1);
    }
    OInternal* in = (OInternal*)calloc((size_t)(N - 1), sizeof(OInternal));
    radix_tree(N, sorted, leaves, in);
    refit(N, leaves, in);
    ONode* nodes = (ONode*)malloc(sizeof(ONode) * (size_t)(2 * N - 1));
    merge(N, leaves, in, nodes);
    if (merged) memcpy(merged, nodes, sizeof(ONode) * (size_t)(2 * N - 1));
    for (int r = 0; r < rounds; ++r) treelet_round(nodes, 2 * N - 1);
    if (final_nodes) memcpy(final_nodes, nodes, sizeof(ONode) * (size_t)(2 * N - 1));
    free(box); free(codes); free(sorted); free(perm); free(leaves); free(in); free(nodes);
    fp_leave(f);
    return 0;
}

/* Runs `rounds` treelet rounds in place on a merged node array (2N-1 records). */
void orc_treelet_rounds(ONode* nodes, int64_t count, int rounds) {
    unsigned f = fp_enter();
    for (int r = 0; r < rounds; ++r) treelet_round(nodes, (int32_t)count);
    fp_leave(f);
}

/* ------------------------------------------------------------- traversal */
static inline int32_t fbits(float x) { int32_t i; memcpy(&i, &x, 4); return i; }
static inline float bitsf(int32_t i) { float x; memcpy(&x, &i, 4); return x; }
static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

/* AABB::intersect, Core/BoundingBox.h:56-74 with fmin_fmax/fmax_fmin
 * (Utils/MathsCommons.h:93-100: vmin/vmax on signed 32-bit float bit patterns). */
static int box_hit(const float* bmin, const float* bmax, const float* o, const float* inv, float* min_dist) {
    float t0[3], t1[3];
    for (int k = 0; k < 3; ++k) {
        t0[k] = (bmin[k] - o[k]) * inv[k];
        t1[k] = (bmax[k] - o[k]) * inv[k];
    }
    float zmin = fminf(t0[2], t1[2]);
    float zmax = fmaxf(t0[2], t1[2]);
    /* fmin_fmax(a,b,c) = int max(int min(a,b), c); fmax_fmin(a,b,c) = int min(int max(a,b), c) */
    float ymm = bitsf(imax(imin(fbits(t0[1]), fbits(t1[1])), fbits(zmin)));
    float maxmin = bitsf(imax(imin(fbits(t0[0]), fbits(t1[0])), fbits(ymm)));
    float yMM = bitsf(imin(imax(fbits(t0[1]), fbits(t1[1])), fbits(zmax)));
    float minmax = bitsf(imin(imax(fbits(t0[0]), fbits(t1[0])), fbits(yMM)));
    if (maxmin <= minmax) {
        if (minmax > 0) {
            *min_dist = fmaxf(0.0f, maxmin);
            return 1;
        }
    }
    *min_dist = -1.0f;
    return 0;
}

/* rayTriangleIntersection, Core/Triangle.h:7-57.  cross/dot contracted as the GPU does:
 * cross.x = fma(a.y, b.z, -(a.z*b.y)); dot = fma(a.z, b.z, fma(a.x, b.x, a.y*b.y)). */
static void cross3(const float* a, const float* b, float* o) {
    o[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
    o[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
    o[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}
static float dot3(const float* a, const float* b) { return fmaf(a[2], b[2], fmaf(a[0], b[0], a[1] * b[1])); }

static int tri_hit(const float* pos, const int32_t* idx, int32_t t, const float* o, const float* d, float* dist,
                   float* uo, float* vo) {
    const float* v0 = pos + 3 * (int64_t)idx[3 * t + 0];
    const float* v1 = pos + 3 * (int64_t)idx[3 * t + 1];
    const float* v2 = pos + 3 * (int64_t)idx[3 * t + 2];
    float e1[3], e2[3], tv[3], pv[3], qv[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = v1[k] - v0[k];
        e2[k] = v2[k] - v0[k];
        tv[k] = o[k] - v0[k];
    }
    cross3(d, e2, pv);
    float det = dot3(e1, pv);
    if (det == 0) return 0;
    det = 1.0f / det;
    float u = dot3(tv, pv) * det;
    if (u < 0.0f || u > 1.0f) return 0;
    cross3(tv, e1, qv);
    float v = dot3(d, qv) * det;
    if (v < 0.0f || (u + v) > 1.0f) return 0;
    float dd = dot3(e2, qv) * det;
    if (dd <= 0.0f) return 0;
    *dist = dd;
    *uo = u;
    *vo = v;
    return 1;
}

/* BVH::intersect, BVH/BVH.h:23-107, over the final node array.  rays: 6 floats each.
 * prim_out: hit triangle (leaf primitiveIndexBegin) or -1.  Uses OpenMP when built with it. */
/* One ray of BVH::intersect (BVH/BVH.h:23-107).  Returns the hit triangle or -1 (-2 on a
 * traversal-stack overflow); writes t/u/v of the hit. */
int32_t orc_closest_one(const ONode* nodes, const float* pos, const int32_t* idx, const float* o, const float* d,
                        float* t_out, float* u_out, float* v_out) {
    float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    int hit = 0;
    float best = 3.402823466e+38f;
    int32_t best_t = -1;
    float bu = 0, bv = 0, md;
    if (box_hit(nodes[0].bmin, nodes[0].bmax, o, inv, &md)) {
        int32_t stack[128];
        int top = 0;
        stack[0] = 0;
        while (top >= 0) {
            int32_t cur = stack[top--];
            const ONode* nd = &nodes[cur];
            if (nd->is_leaf) {
                for (int32_t p = nd->begin; p <= nd->end; ++p) {
                    float dist, u, v;
                    if (tri_hit(pos, idx, p, o, d, &dist, &u, &v)) {
                        if (!hit || dist < best) {
                            hit = 1; best = dist; best_t = p; bu = u; bv = v;
                        }
                    }
                }
            } else {
                float ml, mr;
                box_hit(nodes[nd->left].bmin, nodes[nd->left].bmax, o, inv, &ml);
                box_hit(nodes[nd->right].bmin, nodes[nd->right].bmax, o, inv, &mr);
                int okl = ml >= 0 && ml < best;
                int okr = mr >= 0 && mr < best;
                if (top + 2 >= 128) { hit = 0; best_t = -2; break; } /* stack overflow: flag */
                if (okl && okr) {
                    if (ml > mr) { stack[++top] = nd->left; stack[++top] = nd->right; }
                    else { stack[++top] = nd->right; stack[++top] = nd->left; }
                } else if (okl) stack[++top] = nd->left;
                else if (okr) stack[++top] = nd->right;
            }
        }
    }
    if (t_out) *t_out = best_t >= 0 ? best : INFINITY;
    if (u_out) *u_out = bu;
    if (v_out) *v_out = bv;
    return best_t;
}

/* BVH::intersect over a batch.  rays: 6 floats each.  prim_out: hit triangle (leaf
 * primitiveIndexBegin) or -1.  Uses OpenMP when built with it. */
void orc_trace_closest(const ONode* nodes, const float* pos, const int32_t* idx, const float* rays, int64_t n,
                       int32_t* prim_out, float* t_out, float* u_out, float* v_out) {
    unsigned f = fp_enter();
#pragma omp parallel
    {
        unsigned ff = fp_enter();
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n; ++r) {
            float t, u, v;
            prim_out[r] = orc_closest_one(nodes, pos, idx, rays + 6 * r, rays + 6 * r + 3, &t, &u, &v);
            if (t_out) t_out[r] = t;
            if (u_out) u_out[r] = u;
            if (v_out) v_out[r] = v;
        }
        fp_leave(ff);
    }
    fp_leave(f);
}

/* BVH::testVisibility, BVH/BVH.h:109-189.  limit: per-ray distance limit or NULL;
 * excl: 2 mesh ids per ray (source, target) or NULL; mesh_of_tri: per-triangle mesh id.
 * occluded[r] = 1 when some non-excluded triangle is hit (closer than the limit). */
/* One ray of BVH::testVisibility (BVH/BVH.h:109-189).  Returns 1 when a triangle outside
 * meshes src/dst is hit closer than limit (limit < 0: no limit), 2 on stack overflow. */
int orc_any_one(const ONode* nodes, const float* pos, const int32_t* idx, const int32_t* mesh_of_tri,
                const float* o, const float* d, float limit, int32_t src, int32_t dst) {
    float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    int occ = 0;
    float md;
    box_hit(nodes[0].bmin, nodes[0].bmax, o, inv, &md); /* a miss is only reported */
    int32_t stack[128];
    int top = 0;
    stack[0] = 0;
    while (top >= 0 && !occ) {
        int32_t cur = stack[top--];
        const ONode* nd = &nodes[cur];
        if (nd->is_leaf) {
            for (int32_t p = nd->begin; p <= nd->end; ++p) {
                int32_t mi = mesh_of_tri ? mesh_of_tri[p] : 0;
                if (mi == src || mi == dst) continue;
                float dist, u, v;
                if (tri_hit(pos, idx, p, o, d, &dist, &u, &v)) {
                    if (limit < 0 || dist < limit) { occ = 1; break; }
                }
            }
        } else {
            float ml, mr;
            box_hit(nodes[nd->left].bmin, nodes[nd->left].bmax, o, inv, &ml);
            box_hit(nodes[nd->right].bmin, nodes[nd->right].bmax, o, inv, &mr);
            if (top + 2 >= 128) { occ = 2; break; }
            if (ml >= 0 && mr >= 0) {
                if (ml > mr) { stack[++top] = nd->left; stack[++top] = nd->right; }
                else { stack[++top] = nd->right; stack[++top] = nd->left; }
            } else if (ml >= 0) stack[++top] = nd->left;
            else if (mr >= 0) stack[++top] = nd->right;
        }
    }
    return occ;
}

/* BVH::testVisibility over a batch.  limit: per-ray distance limit or NULL; excl: 2 mesh
 * ids per ray (source, target) or NULL; mesh_of_tri: per-triangle mesh id.  occluded[r] = 1
 * when some non-excluded triangle is hit (closer than the limit). */
void orc_trace_any(const ONode* nodes, const float* pos, const int32_t* idx, const int32_t* mesh_of_tri,
                   const float* rays, const float* limit, const int32_t* excl, int64_t n, uint8_t* occluded) {
    unsigned f = fp_enter();
#pragma omp parallel
    {
        unsigned ff = fp_enter();
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n; ++r) {
            int32_t src = excl ? excl[2 * r] : -1, dst = excl ? excl[2 * r + 1] : -1;
            occluded[r] = (uint8_t)orc_any_one(nodes, pos, idx, mesh_of_tri, rays + 6 * r, rays + 6 * r + 3,
                                               limit ? limit[r] : -1.0f, src, dst);
        }
        fp_leave(ff);
    }
    fp_leave(f);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
