// Test infrastructure: golden/timing harness around the reference's own CUDA code.
//
// This translation unit is compiled by oracle/build_ref.sh inside a symlink farm
// (oracle/_ref/src) whose BVH/, Utils/ and Core/{BoundingBox,Triangle,Ray,
// VisibilityTest}.h entries point at the reference sources where they lie, and whose
// Core/{TriangleMesh,IntersectionResult}.h point at the shims in oracle/ref_shim.
// It includes the reference's BVH/BVH.cu and BVH/Optimization.cu verbatim and
// replays BVH::build (BVH/BVH.cu:317-370) stage by stage, so that intermediate
// results (Morton codes, sorted order, node arrays before and after the treelet
// rounds) can be dumped and every stage timed with CUDA events.  Traversal calls
// the verbatim BVH::intersect / BVH::testVisibility (BVH/BVH.h:23-189).
//
// Only tests/ (golden generation, live parity) and the reference-timing script
// load the resulting library.  Nothing in the product links it.

#include "../BVH/BVH.cu"
#include "../BVH/Optimization.cu"

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct RefScene {
    int ntri = 0;
    int nvert = 0;
    float3* d_pos = nullptr;
    int3* d_idx = nullptr;
    float2* d_tex = nullptr;
    TriangleMesh* d_meshes = nullptr;
    Triangle* d_tris = nullptr;
    BVH* bvh = nullptr;
    int depth = 0;
    int id_mode = 0;
};

#define RCHK(x)                                                     \
    do {                                                            \
        cudaError_t e_ = (x);                                       \
        if (e_ != cudaSuccess) {                                    \
            fprintf(stderr, "ref_harness: %s at %s:%d\n",           \
                    cudaGetErrorString(e_), __FILE__, __LINE__);    \
            return -1;                                              \
        }                                                           \
    } while (0)

}  // namespace

// Plain, packed mirror of BVHRestructureNode (BVH/BVHNode.h:50-68) for dumps.
struct RefRNodeOut {
    float bmin[3];
    float bmax[3];
    int begin, end, left, right, parent, is_leaf;
    float area, cost;
};

static void dump_rnodes(const std::vector<BVHRestructureNode>& h, RefRNodeOut* out) {
    for (size_t i = 0; i < h.size(); ++i) {
        const BVHRestructureNode& n = h[i];
        out[i].bmin[0] = n.box.minimum.x; out[i].bmin[1] = n.box.minimum.y; out[i].bmin[2] = n.box.minimum.z;
        out[i].bmax[0] = n.box.maximum.x; out[i].bmax[1] = n.box.maximum.y; out[i].bmax[2] = n.box.maximum.z;
        out[i].begin = n.primitiveIndexBegin;
        out[i].end = n.primitiveIndexEnd;
        out[i].left = n.leftChild;
        out[i].right = n.rightChild;
        out[i].parent = n.parent;
        out[i].is_leaf = n.isLeaf ? 1 : 0;
        out[i].area = n.surfaceArea;
        out[i].cost = n.cost;
    }
}

static int tree_depth(const std::vector<BVHNode>& nodes) {
    if (nodes.empty()) return 0;
    std::vector<std::pair<int, int>> st;
    st.push_back({0, 0});
    int best = 0;
    size_t guard = 0;
    while (!st.empty()) {
        auto [n, d] = st.back();
        st.pop_back();
        if (++guard > 4 * nodes.size() + 8) return 1 << 30;  // malformed tree
        if (n < 0 || n >= (int)nodes.size()) return 1 << 30;
        best = d > best ? d : best;
        if (!nodes[n].isLeaf) {
            st.push_back({nodes[n].leftChild, d + 1});
            st.push_back({nodes[n].rightChild, d + 1});
        }
    }
    return best;
}

// Builds the BVH exactly as BVH::build does and keeps the scene for traversal.
// pos: nvert*3 floats; idx: ntri*3 ints (global vertex indices); mesh_of_tri: ntri ints
// (the Triangle::meshIndex of each triangle, in the global order of
// TriangleMesh::copyTrianglesToScene, Core/TriangleMesh.cu:190-195).
// id_mode=1 gives every triangle its own mesh record whose `prim` pointer encodes
// the triangle index, so that BVH::intersect's result identifies the hit triangle;
// the arithmetic on positions/indices is unchanged.  id_mode=0 uses one mesh record
// per mesh id (the reference's own layout; used for timing).
// scene_bounds: 6 floats or NULL (then the host fold of Core/Scene.cu:131-135).
// Any output pointer may be NULL.  stage_ms (8 floats): leaf boxes, Morton, sort,
// radix tree, bounds, merge, treelet rounds (total), final copy.
extern "C" int ref_build(const float* pos, int nvert, const int* idx, const int* mesh_of_tri, int ntri,
                         int id_mode, const float* scene_bounds, int rounds,
                         unsigned long long* codes_unsorted, unsigned long long* codes_sorted,
                         int* perm_sorted, RefRNodeOut* nodes_merged, RefRNodeOut* nodes_final_r,
                         float* bounds_out, float* stage_ms, void** handle_out) {
    if (ntri < 2 || nvert < 1) return -3;
    // The reference's treelet kernel (optimizeBVHImpl, BVH/Optimization.cu:467-507) raised
    // an illegal memory access on the B200 on a 34-triangle input.  Reading the code, the
    // 6-leaf step shifts by a negative amount when emptyBit == 6 (:232,
    // consequtiveBits(5-emptyBit)), which is undefined behaviour.  It is never launched
    // again: this harness refuses any request with treelet rounds.
    if (rounds != 0) return -4;
    RefScene* s = new RefScene();
    s->ntri = ntri;
    s->nvert = nvert;
    s->id_mode = id_mode;

    RCHK(cudaMalloc(&s->d_pos, sizeof(float3) * nvert));
    RCHK(cudaMalloc(&s->d_idx, sizeof(int3) * ntri));
    RCHK(cudaMalloc(&s->d_tex, sizeof(float2) * nvert));
    RCHK(cudaMemcpy(s->d_pos, pos, sizeof(float3) * nvert, cudaMemcpyHostToDevice));
    RCHK(cudaMemcpy(s->d_idx, idx, sizeof(int3) * ntri, cudaMemcpyHostToDevice));
    RCHK(cudaMemset(s->d_tex, 0, sizeof(float2) * nvert));

    int max_mesh = 0;
    for (int i = 0; i < ntri; ++i) max_mesh = mesh_of_tri[i] > max_mesh ? mesh_of_tri[i] : max_mesh;
    int nmesh = id_mode ? ntri : max_mesh + 1;
    std::vector<TriangleMesh> hmesh(nmesh);
    for (int m = 0; m < nmesh; ++m) {
        hmesh[m].trianglesCount = ntri;
        hmesh[m].verticesCount = nvert;
        hmesh[m].positions.gpu.data = s->d_pos;
        hmesh[m].indices.gpu.data = s->d_idx;
        hmesh[m].normals.gpu.data = s->d_pos;
        hmesh[m].texCoords.gpu.data = s->d_tex;
        hmesh[m].positions.cpu.data = (float3*)pos;
        hmesh[m].indices.cpu.data = (int3*)idx;
        hmesh[m].meshIndex = id_mode ? mesh_of_tri[m] : m;
        hmesh[m].prim = id_mode ? (Primitive*)(uintptr_t)(m + 1) : nullptr;
    }
    RCHK(cudaMalloc(&s->d_meshes, sizeof(TriangleMesh) * nmesh));
    RCHK(cudaMemcpy(s->d_meshes, hmesh.data(), sizeof(TriangleMesh) * nmesh, cudaMemcpyHostToDevice));

    std::vector<Triangle> htri;
    htri.reserve(ntri);
    for (int i = 0; i < ntri; ++i) {
        Triangle t(mesh_of_tri[i], i);
        t.mesh = &hmesh[id_mode ? i : mesh_of_tri[i]];
        htri.push_back(t);
    }
    AABB sceneBounds;
    if (scene_bounds) {
        sceneBounds.minimum = make_float3(scene_bounds[0], scene_bounds[1], scene_bounds[2]);
        sceneBounds.maximum = make_float3(scene_bounds[3], scene_bounds[4], scene_bounds[5]);
    } else {
        sceneBounds = htri[0].getBoundingBox();
        for (int i = 1; i < ntri; ++i) sceneBounds = unionBoxes(sceneBounds, htri[i].getBoundingBox());
    }
    if (bounds_out) {
        bounds_out[0] = sceneBounds.minimum.x; bounds_out[1] = sceneBounds.minimum.y; bounds_out[2] = sceneBounds.minimum.z;
        bounds_out[3] = sceneBounds.maximum.x; bounds_out[4] = sceneBounds.maximum.y; bounds_out[5] = sceneBounds.maximum.z;
    }
    for (int i = 0; i < ntri; ++i) htri[i].mesh = s->d_meshes + (id_mode ? i : mesh_of_tri[i]);
    RCHK(cudaMalloc(&s->d_tris, sizeof(Triangle) * ntri));
    RCHK(cudaMemcpy(s->d_tris, htri.data(), sizeof(Triangle) * ntri, cudaMemcpyHostToDevice));
    RCHK(cudaDeviceSynchronize());

    cudaEvent_t ev[9];
    for (int i = 0; i < 9; ++i) cudaEventCreate(&ev[i]);

    // --- replay of BVH::build, BVH/BVH.cu:317-370 ---
    int primitivesCount = ntri;
    s->bvh = new BVH(primitivesCount);
    BVH& bvh = *s->bvh;
    GpuArray<BVHLeafNode> leaves(primitivesCount);
    int numThreadsPrimitives = min(primitivesCount, MAX_THREADS_PER_BLOCK);
    int numBlocksPrimitives = divUp(primitivesCount, numThreadsPrimitives);
    GpuArray<MortonType> leafMortonCodes(primitivesCount);
    GpuArray<BVHInternalNode> internals(primitivesCount - 1);
    GpuArray<BVHRestructureNode> restructureNodes(bvh.nodes.N, false);
    RCHK(cudaDeviceSynchronize());

    cudaEventRecord(ev[0]);
    fillLeafBoundingBoxes<<<numBlocksPrimitives, numThreadsPrimitives>>>(s->d_tris, primitivesCount, leaves.data);
    cudaEventRecord(ev[1]);
    fillLeafMortonCodes<<<numBlocksPrimitives, numThreadsPrimitives>>>(s->d_tris, primitivesCount, leaves.data,
                                                                       leafMortonCodes.data, sceneBounds);
    cudaEventRecord(ev[2]);
    RCHK(cudaDeviceSynchronize());
    if (codes_unsorted)
        RCHK(cudaMemcpy(codes_unsorted, leafMortonCodes.data, sizeof(MortonType) * primitivesCount,
                        cudaMemcpyDeviceToHost));
    cudaEventRecord(ev[2]);
    thrust::stable_sort_by_key(thrust::device, leafMortonCodes.data, leafMortonCodes.data + primitivesCount,
                               leaves.data, thrust::less<MortonType>());
    cudaEventRecord(ev[3]);
    int numThreadsInternals = min(primitivesCount - 1, MAX_THREADS_PER_BLOCK);
    int numBlocksInternals = divUp(primitivesCount - 1, numThreadsPrimitives);
    buildRadixTree<<<numBlocksInternals, numThreadsInternals>>>(primitivesCount, leafMortonCodes.data, leaves.data,
                                                                 internals.data);
    cudaEventRecord(ev[4]);
    computeBounds<<<numBlocksPrimitives, numThreadsPrimitives>>>(primitivesCount, leaves.data, internals.data);
    cudaEventRecord(ev[5]);
    mergeNodesArray<<<numBlocksInternals, numThreadsInternals>>>(primitivesCount, leaves.data, internals.data,
                                                                 restructureNodes.data);
    cudaEventRecord(ev[6]);
    RCHK(cudaDeviceSynchronize());
    RCHK(cudaGetLastError());

    if (codes_sorted)
        RCHK(cudaMemcpy(codes_sorted, leafMortonCodes.data, sizeof(MortonType) * primitivesCount,
                        cudaMemcpyDeviceToHost));
    if (perm_sorted) {
        std::vector<BVHLeafNode> hl = leaves.toVector();
        for (int i = 0; i < primitivesCount; ++i) perm_sorted[i] = hl[i].primitiveIndexBegin;
    }
    if (nodes_merged) dump_rnodes(restructureNodes.toVector(), nodes_merged);

    cudaEventRecord(ev[6]);
    optimizeBVH(primitivesCount, restructureNodes, rounds);
    cudaEventRecord(ev[7]);
    int numBlocksAllNodes, numThreadsAllNodes;
    setNumBlocksThreads(bvh.nodes.N, numBlocksAllNodes, numThreadsAllNodes);
    copyToBVH<<<numBlocksAllNodes, numThreadsAllNodes>>>(bvh.nodes.N, restructureNodes.data, bvh.nodes.data);
    cudaEventRecord(ev[8]);
    RCHK(cudaDeviceSynchronize());
    RCHK(cudaGetLastError());

    if (stage_ms) {
        for (int i = 0; i < 8; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
    }
    for (int i = 0; i < 9; ++i) cudaEventDestroy(ev[i]);

    if (nodes_final_r) dump_rnodes(restructureNodes.toVector(), nodes_final_r);
    s->depth = tree_depth(bvh.nodes.toVector());
    *handle_out = s;
    return 0;
}

// Final BVHNode array (BVH/BVHNode.h:8-21) as a plain 44-byte record.
struct RefNodeOut {
    float bmin[3];
    float bmax[3];
    int begin, end, left, right, is_leaf;
};

extern "C" int ref_export_nodes(void* h, RefNodeOut* out) {
    RefScene* s = (RefScene*)h;
    std::vector<BVHNode> n = s->bvh->nodes.toVector();
    for (size_t i = 0; i < n.size(); ++i) {
        out[i].bmin[0] = n[i].box.minimum.x; out[i].bmin[1] = n[i].box.minimum.y; out[i].bmin[2] = n[i].box.minimum.z;
        out[i].bmax[0] = n[i].box.maximum.x; out[i].bmax[1] = n[i].box.maximum.y; out[i].bmax[2] = n[i].box.maximum.z;
        out[i].begin = n[i].primitiveIndexBegin;
        out[i].end = n[i].primitiveIndexEnd;
        out[i].left = n[i].leftChild;
        out[i].right = n[i].rightChild;
        out[i].is_leaf = n[i].isLeaf ? 1 : 0;
    }
    return 0;
}

extern "C" int ref_tree_depth(void* h) { return ((RefScene*)h)->depth; }

// Replaces the reference BVH's node array with `nodes` (2N-1 records), so that the
// reference's verbatim traversal can be run on a given tree (a race-free LBVH, or a
// tree after treelet rounds computed elsewhere).  Returns -2 for a malformed tree.
extern "C" int ref_load_nodes(void* h, const RefNodeOut* nodes, int count) {
    RefScene* s = (RefScene*)h;
    if (count != s->bvh->nodes.N) return -1;
    std::vector<BVHNode> v((size_t)count);
    for (int i = 0; i < count; ++i) {
        memset(&v[i], 0, sizeof(BVHNode));
        v[i].box.minimum = make_float3(nodes[i].bmin[0], nodes[i].bmin[1], nodes[i].bmin[2]);
        v[i].box.maximum = make_float3(nodes[i].bmax[0], nodes[i].bmax[1], nodes[i].bmax[2]);
        v[i].primitiveIndexBegin = nodes[i].begin;
        v[i].primitiveIndexEnd = nodes[i].end;
        v[i].leftChild = nodes[i].left;
        v[i].rightChild = nodes[i].right;
        v[i].isLeaf = nodes[i].is_leaf != 0;
        if (v[i].isLeaf && (nodes[i].begin < 0 || nodes[i].end >= s->ntri || nodes[i].begin > nodes[i].end)) return -2;
    }
    int d = tree_depth(v);
    if (d >= (1 << 30)) return -2;
    RCHK(cudaMemcpy(s->bvh->nodes.data, v.data(), sizeof(BVHNode) * (size_t)count, cudaMemcpyHostToDevice));
    s->depth = d;
    return 0;
}

__global__ void refClosestKernel(BVH bvh, Triangle* prims, const float* rays, int n, int id_mode, int* prim_out,
                                 float* t_out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Ray r;
    r.origin = make_float3(rays[6 * i + 0], rays[6 * i + 1], rays[6 * i + 2]);
    r.direction = make_float3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    IntersectionResult res;
    bool hit = bvh.intersect(res, r, prims);
    if (prim_out) prim_out[i] = hit ? (id_mode ? (int)((uintptr_t)res.primitive - 1) : 0) : -1;
    if (t_out) t_out[i] = hit ? res.distance : __int_as_float(0x7f800000);
}

__global__ void refAnyKernel(BVH bvh, Triangle* prims, const float* rays, const float* limit, const int* excl,
                             int n, unsigned char* occluded) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    VisibilityTest test;
    test.ray.origin = make_float3(rays[6 * i + 0], rays[6 * i + 1], rays[6 * i + 2]);
    test.ray.direction = make_float3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    if (limit) test.setDistanceLimit(limit[i]);
    test.sourceMeshIndex = excl ? excl[2 * i] : -1;
    test.targetMeshIndex = excl ? excl[2 * i + 1] : -1;
    occluded[i] = bvh.testVisibility(test, prims) ? 0 : 1;
}

// The reference's traversal keeps a fixed `int stack[64]` with no overflow check
// (BVH/BVH.h:41, :122).  The stack never holds more than depth+1 entries, so trees
// deeper than 62 are refused here instead of being traced.
static const int kMaxSafeDepth = 62;

// rays: n * 6 floats (origin, direction) on the host.  Outputs on the host.
// ms_out: kernel time of `reps` back-to-back launches (average), CUDA events.
extern "C" int ref_trace_closest(void* h, const float* rays, int n, int reps, int* prim_out, float* t_out,
                                 float* ms_out) {
    RefScene* s = (RefScene*)h;
    if (s->depth > kMaxSafeDepth) return -2;
    float* d_rays;
    int* d_prim;
    float* d_t;
    RCHK(cudaMalloc(&d_rays, sizeof(float) * 6 * (size_t)n));
    RCHK(cudaMalloc(&d_prim, sizeof(int) * (size_t)n));
    RCHK(cudaMalloc(&d_t, sizeof(float) * (size_t)n));
    RCHK(cudaMemcpy(d_rays, rays, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice));
    int threads = min(n, MAX_THREADS_PER_BLOCK);
    int blocks = divUp(n, threads);
    refClosestKernel<<<blocks, threads>>>(s->bvh->getCopyForKernel(), s->d_tris, d_rays, n, s->id_mode, d_prim, d_t);
    RCHK(cudaDeviceSynchronize());
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    if (reps < 1) reps = 1;
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r)
        refClosestKernel<<<blocks, threads>>>(s->bvh->getCopyForKernel(), s->d_tris, d_rays, n, s->id_mode, d_prim,
                                              d_t);
    cudaEventRecord(b);
    RCHK(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms_out) *ms_out = ms / reps;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    RCHK(cudaGetLastError());
    if (prim_out) RCHK(cudaMemcpy(prim_out, d_prim, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    if (t_out) RCHK(cudaMemcpy(t_out, d_t, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(d_rays);
    cudaFree(d_prim);
    cudaFree(d_t);
    return 0;
}

// limit: n floats or NULL (no distance limit); excl: 2n ints (source, target mesh) or NULL (-1, -1).
extern "C" int ref_trace_any(void* h, const float* rays, const float* limit, const int* excl, int n, int reps,
                             unsigned char* occluded, float* ms_out) {
    RefScene* s = (RefScene*)h;
    if (s->depth > kMaxSafeDepth) return -2;
    float *d_rays, *d_lim = nullptr;
    int* d_excl = nullptr;
    unsigned char* d_occ;
    RCHK(cudaMalloc(&d_rays, sizeof(float) * 6 * (size_t)n));
    RCHK(cudaMemcpy(d_rays, rays, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice));
    if (limit) {
        RCHK(cudaMalloc(&d_lim, sizeof(float) * (size_t)n));
        RCHK(cudaMemcpy(d_lim, limit, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
    }
    if (excl) {
        RCHK(cudaMalloc(&d_excl, sizeof(int) * 2 * (size_t)n));
        RCHK(cudaMemcpy(d_excl, excl, sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice));
    }
    RCHK(cudaMalloc(&d_occ, (size_t)n));
    int threads = min(n, MAX_THREADS_PER_BLOCK);
    int blocks = divUp(n, threads);
    refAnyKernel<<<blocks, threads>>>(s->bvh->getCopyForKernel(), s->d_tris, d_rays, d_lim, d_excl, n, d_occ);
    RCHK(cudaDeviceSynchronize());
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    if (reps < 1) reps = 1;
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r)
        refAnyKernel<<<blocks, threads>>>(s->bvh->getCopyForKernel(), s->d_tris, d_rays, d_lim, d_excl, n, d_occ);
    cudaEventRecord(b);
    RCHK(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms_out) *ms_out = ms / reps;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    RCHK(cudaGetLastError());
    RCHK(cudaMemcpy(occluded, d_occ, (size_t)n, cudaMemcpyDeviceToHost));
    cudaFree(d_rays);
    cudaFree(d_lim);
    cudaFree(d_excl);
    cudaFree(d_occ);
    return 0;
}

extern "C" void ref_free(void* h) {
    RefScene* s = (RefScene*)h;
    if (!s) return;
    delete s->bvh;
    cudaFree(s->d_pos);
    cudaFree(s->d_idx);
    cudaFree(s->d_tex);
    cudaFree(s->d_meshes);
    cudaFree(s->d_tris);
    delete s;
}
