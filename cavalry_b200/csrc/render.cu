// Wavefront path tracer for sm_100a: the generate / extend / lighting (shadow) / material
// evaluation / next-ray stages of the reference's PathTracingIntegrator
// (Integrators/PathTracingIntegrator.cu:95-425), with queues compacted by warp-aggregated
// atomics and every ray query going through the persistent traversal kernels of trace.cu.
//
// Sampling follows the reference exactly so that a render with the same sample count uses
// the same random numbers per path: scrambled Halton (Samplers/HaltonSampler.h:13-76,
// HaltonSampler.cu:14-67; the permutation tables are built on the host with the C
// library's srand/rand, as the reference does), camera samples (Core/Sampler.cu:29-51),
// and the per-bounce dimension budget of computeLighting / genNextRay (randInt for the
// light, an unused rand4, the light-triangle sample, then Russian roulette after depth 3
// and a BSDF rand2).  Shading is FP32 and restates the reference's BSDFs: Lambertian
// (BSDFs/Lambertian.h), plastic = Lambertian + GGX microfacet reflection with Schlick
// Fresnel (BSDFs/PlasticBSDF.h, Microfacet.h, MicrofacetDistribution.h, Fresnel.h),
// specular glass (BSDFs/Specular.h) and mirror (BSDFs/MirrorBSDF.h); area lights are the
// reference's DiffuseAreaLight (Lights/DiffuseAreaLight.h, Core/TriangleMesh.h:110-232).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "render_common.cuh"

namespace cav {
namespace {

// intersectScene + computeLighting + genNextRay (PathTracingIntegrator.cu:95-225) for one
// bounce; the shadow ray is traced in a separate any-hit launch and its contribution added
// by k_add_direct (evalMaterial, :227-249, is folded in here).
// n_dev (or null): the queue size read from device memory (graph-replayed bounces)
// 4 blocks per SM (64 registers, a few hundred bytes spilled): shading waits on dependent
// loads (hit, triangle, material, texture), so resident warps pay more than registers.
// Measured on the 5.24M-triangle icosphere render (1920x1080, 64 spp, depth 8): 129.9 ms of
// shading at 96 registers, 105.3 at 80, 96.4 at 64.
__global__ void __launch_bounds__(kThreads, 4) k_shade(DevScene S, int depth, int dim0, int64_t n, Paths P, Queues Q,
                        const uint32_t* n_dev = nullptr) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev) n = *n_dev;
    bool valid = j < n;
    int path = valid ? Q.active[j] : 0;
    int prim = valid ? Q.hit_prim[j] : -1;
    bool hit = valid && prim >= 0;
    bool emit_shadow = false, cont = false;
    cav_ray shadow{}, next{};
    float limit = 0.f;
    int2 excl = make_int2(-1, -1);
    f3 contrib = mk(0, 0, 0);
    f3 thr = mk(0, 0, 0);
    float next_pdf = 0.f;
    bool next_delta = false;
    if (hit) {
        const cav_ray r = Q.rays[j];
        f3 ro = mk(r.ox, r.oy, r.oz), rd = mk(r.dx, r.dy, r.dz);
        float t = Q.hit_t[j];
        float u = Q.hit_uv[2 * j], v = Q.hit_uv[2 * j + 1];
        uint64_t index = P.sample_index[path];
        thr = ld3(P.throughput + 3 * path);
        f3 res = ld3(P.result + 3 * path);
        const int mesh = S.tri_mesh[prim];
        const RMesh& M = S.meshes[mesh];
        f3 pos = ro + t * rd;  // Ray::positionAtDistance
        f3 nrm = tri_normal(S, M, prim, u, v);
        // ---- emission at the hit (computeLighting :190-205)
        if (M.light >= 0) {
            const RLight& L = S.lights[M.light];
            f3 Le = dot3(rd, nrm) >= 0 ? mk(0, 0, 0) : ld3(L.L);
            if (P.delta[path]) {
                res = res + Le * thr;
            } else if (depth > 0) {
                float light_pdf = light_surface_pdf(S.meshes[L.mesh], ro, pos, nrm);
                float w = mis_power(P.mat_pdf[path], light_pdf);
                if (isfinite(w)) res = res + Le * thr * w;
            }
        }
        P.result[3 * path] = res.x;
        P.result[3 * path + 1] = res.y;
        P.result[3 * path + 2] = res.z;
        const Bsdf B = material_bsdf(S, S.mats[M.material], prim, u, v);
        const Frame fr = make_frame(nrm);
        const f3 wo_world = rd * -1.f;
        const f3 wo = to_local(fr, wo_world);
        // ---- light sample (computeLighting :207-224)
        int dim = dim0;
        int li = halton_int(S.halton, index, dim, S.n_lights);
        dim += 4;  // rand4, drawn and unused by the reference
        const LightSample ls = sample_light(S, S.lights[li], pos, index, dim);
        const float light_pdf = ls.pdf;
        const f3 dir = ls.dir;
        if (isfinite(light_pdf)) {
            f3 wi = to_local(fr, dir);
            float w = S.direct ? 1.f : mis_power(light_pdf, B.pdf(wi, wo));
            float cosine = fabsf(dot3(dir, nrm));
            f3 mult = thr * (float)S.n_lights / light_pdf;
            contrib = ls.incident * B.eval(wi, wo) * cosine * mult * w;
            if (!all_zero(contrib)) {
                emit_shadow = true;
                shadow = cav_ray{pos.x, pos.y, pos.z, 0.f, dir.x, dir.y, dir.z, INFINITY};
                limit = ls.dist;
                excl = make_int2(mesh, ls.target);
            }
        }
        // ---- continuation (genNextRay :124-171)
        dim = dim0 + S.cont_dim;
        bool alive = !S.direct;
        if (depth > 3) {
            float q = 1;
            q = fminf(q, 1 - thr.x);
            q = fminf(q, 1 - thr.y);
            q = fminf(q, 1 - thr.z);
            q = fmaxf(q, 0.05f);
            if (halton(S.halton, index, dim) < q) alive = false;
            else thr = thr / (1.f - q);
        }
        if (alive) {
            float u0 = halton(S.halton, index, dim);
            float u1 = halton(S.halton, index, dim);
            f3 wi;
            float p = 0.f;
            f3 f = B.sample(u0, u1, wo, wi, p);
            f3 nd = to_world(fr, wi);
            f3 no = pos + nd * 0.001f;
            if (all_zero(f)) thr = mk(0, 0, 0);
            else thr = thr * f * fabsf(dot3(nd, nrm)) / p;
            next_pdf = p;
            next_delta = B.is_delta();
            // A path whose throughput is exactly zero adds nothing on later bounces; the
            // reference traces it anyway, this queue drops it.
            if (!all_zero(thr)) {
                cont = true;
                next = cav_ray{no.x, no.y, no.z, 0.f, nd.x, nd.y, nd.z, INFINITY};
            }
        }
    }
    if (valid && !hit && S.env >= 0) {  // intersectScene :111-116: the environment, no MIS weight
        const cav_ray r = Q.rays[j];
        const f3 e = env_eval(S, S.lights[S.env], mk(r.dx, r.dy, r.dz)) * ld3(P.throughput + 3 * path);
        P.result[3 * path] += e.x;
        P.result[3 * path + 1] += e.y;
        P.result[3 * path + 2] += e.z;
    }
    uint32_t ks = warp_append(Q.counters + 1, emit_shadow);
    if (emit_shadow) {
        Q.shadow_rays[ks] = shadow;
        Q.shadow_limit[ks] = limit;
        reinterpret_cast<int2*>(Q.shadow_excl)[ks] = excl;
        Q.shadow_path[ks] = path;
        Q.shadow_contrib[3 * ks] = contrib.x;
        Q.shadow_contrib[3 * ks + 1] = contrib.y;
        Q.shadow_contrib[3 * ks + 2] = contrib.z;
    }
    uint32_t kn = warp_append(Q.counters + 0, cont);
    if (cont) {
        Q.next_active[kn] = path;
        Q.next_rays[kn] = next;
        P.throughput[3 * path] = thr.x;
        P.throughput[3 * path + 1] = thr.y;
        P.throughput[3 * path + 2] = thr.z;
        P.mat_pdf[path] = next_pdf;
        P.delta[path] = next_delta ? 1 : 0;
    }
}

// evalMaterial's accumulation for unoccluded shadow rays.  The paths of one bounce are
// distinct, so plain read-modify-write is race free.
__global__ void k_add_direct(int64_t n, Paths P, Queues Q, const uint32_t* n_dev = nullptr) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev) n = *n_dev;
    if (k >= n) return;
    if (Q.shadow_occ[k] != 0) return;
    int path = Q.shadow_path[k];
    P.result[3 * path] += Q.shadow_contrib[3 * k];
    P.result[3 * path + 1] += Q.shadow_contrib[3 * k + 1];
    P.result[3 * path + 2] += Q.shadow_contrib[3 * k + 2];
}

// Permutation tables of HaltonSampler.cu:14-67: the first 1024 primes; one Fisher-Yates
// shuffle per prime driven by the C library's rand() after srand(533799).
void build_halton_tables(std::vector<uint32_t>& primes, std::vector<uint32_t>& start, std::vector<uint16_t>& perms) {
    primes.clear();
    primes.push_back(2);
    for (uint32_t i = 3; primes.size() < (size_t)kPrimes; ++i) {
        bool is_prime = true;
        for (uint32_t p : primes) {
            if (p * p > i) break;
            if (i % p == 0) {
                is_prime = false;
                break;
            }
        }
        if (is_prime) primes.push_back(i);
    }
    start.assign(primes.size(), 0);
    size_t size = 0;
    for (size_t k = 0; k < primes.size(); ++k) {
        start[k] = (uint32_t)size;
        size += primes[k];
    }
    perms.assign(size, 0);
    std::srand(533799);
    for (size_t k = 0; k < primes.size(); ++k) {
        uint32_t p = primes[k];
        std::vector<uint16_t> v(p);
        for (uint32_t j = 0; j < p; ++j) v[j] = (uint16_t)j;
        for (int m = (int)p - 1; m > 0; --m) std::swap(v[m], v[std::rand() % (m + 1)]);
        std::memcpy(&perms[start[k]], v.data(), p * sizeof(uint16_t));
    }
}

}  // namespace
}  // namespace cav

namespace cav {

// The Halton tables depend only on the reference's fixed srand(533799): the host tables are
// computed once per process (std::rand is process-wide state, so never from two threads at
// once) and copied to the device once per context; every scene of the context shares them.
struct HaltonTables {
    std::vector<uint32_t> primes, start;
    std::vector<uint16_t> perms;
};
static const HaltonTables& halton_tables() {
    static std::once_flag once;
    static HaltonTables t;
    std::call_once(once, [] { build_halton_tables(t.primes, t.start, t.perms); });
    return t;
}

static cav_status ctx_halton(cav_ctx* ctx, cav_scene* sc) {
    std::lock_guard<std::mutex> lk(ctx->halton_mu);
    if (!ctx->d_halton_perms) {
        const HaltonTables& t = halton_tables();
        void *a = nullptr, *b = nullptr, *c = nullptr;
        if (cudaMalloc(&a, t.primes.size() * 4) != cudaSuccess || cudaMalloc(&b, t.start.size() * 4) != cudaSuccess ||
            cudaMalloc(&c, t.perms.size() * 2) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(a);
            cudaFree(b);
            return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "Halton tables: device allocation failed");
        }
        CAV_CUDA(ctx, cudaMemcpy(a, t.primes.data(), t.primes.size() * 4, cudaMemcpyHostToDevice));
        CAV_CUDA(ctx, cudaMemcpy(b, t.start.data(), t.start.size() * 4, cudaMemcpyHostToDevice));
        CAV_CUDA(ctx, cudaMemcpy(c, t.perms.data(), t.perms.size() * 2, cudaMemcpyHostToDevice));
        ctx->d_halton_primes = (uint32_t*)a;
        ctx->d_halton_start = (uint32_t*)b;
        ctx->d_halton_perms = (uint16_t*)c;
    }
    sc->d_primes = ctx->d_halton_primes;
    sc->d_perm_start = ctx->d_halton_start;
    sc->d_perms = ctx->d_halton_perms;
    return CAV_OK;
}

// Device bytes a scene takes once uploaded and built (geometry, the tree, the build's peak
// scratch): the server's admission estimate for jobs that bring their own scene.
size_t scene_device_bytes(const cavpbrt::Scene& D) {
    size_t v = 0, t = 0, uv = 0, nrm = 0;
    for (const auto& m : D.meshes) {
        v += m.positions.size() / 3;
        t += m.indices.size() / 3;
        uv += m.uvs.size() / 2;
        nrm += m.normals.size() / 3;
    }
    size_t b = 12 * v + 16 * t + (nrm ? 12 * v : 0) + (uv ? 8 * v : 0) + 4096 * 4;
    for (const auto& tx : D.textures) b += (size_t)(tx.is_float ? 16 : 4) * tx.width * tx.height;
    b += bvh_arena_bytes((int64_t)std::max<size_t>(t, 2)) + 96 * t;  // tree + build scratch
    return b;
}

// Uploads a parsed scene (geometry, materials, lights, textures) without building its BVH.
// async: device arrays are stream-ordered allocations and copies on `s` (the caller builds
// and renders on `s` and releases with scene_release_async); else plain, synchronous ones.
cav_status scene_upload(cav_ctx* ctx, cavpbrt::Scene&& desc, cudaStream_t stream, bool async, cav_scene** out) {
    auto sc = new cav_scene();
    sc->device = ctx->device;
    sc->async_mem = async;
    sc->desc = std::move(desc);
    auto upload = [&](void** dst, const void* src, size_t bytes) -> cav_status {
        CAV_CUDA(ctx, dev_alloc(ctx, dst, bytes > 0 ? bytes : 16, stream, async));
        if (bytes) {
            if (async) CAV_CUDA(ctx, cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream));
            else CAV_CUDA(ctx, cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        }
        return CAV_OK;
    };
    const cavpbrt::Scene& D = sc->desc;
    std::vector<float> pos, nrm;
    std::vector<int32_t> idx, tri_mesh;
    std::vector<RMesh> meshes;
    bool any_normals = false;
    for (const auto& m : D.meshes) any_normals |= !m.normals.empty();
    for (size_t mi = 0; mi < D.meshes.size(); ++mi) {
        const auto& m = D.meshes[mi];
        RMesh rm{};
        rm.first_tri = (int32_t)(idx.size() / 3);
        rm.tri_count = (int32_t)(m.indices.size() / 3);
        rm.has_normals = m.normals.empty() ? 0 : 1;
        rm.reverse = m.reverse_orientation ? 1 : 0;
        rm.material = m.material;
        rm.light = m.light;
        rm.shape = m.shape;
        for (int k = 0; k < 4; ++k) rm.sphere[k] = m.sphere[k];
        // TriangleMesh::computeArea (Core/TriangleMesh.cu:189-199): float sum of half cross lengths
        float area = 0.f;
        for (size_t t = 0; t < m.indices.size() / 3; ++t) {
            const float* p0 = &m.positions[3 * m.indices[3 * t]];
            const float* p1 = &m.positions[3 * m.indices[3 * t + 1]];
            const float* p2 = &m.positions[3 * m.indices[3 * t + 2]];
            float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
            float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            area += std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) * 0.5f;
        }
        rm.area = area;
        int32_t vbase = (int32_t)(pos.size() / 3);
        pos.insert(pos.end(), m.positions.begin(), m.positions.end());
        if (any_normals) {
            if (m.normals.empty()) nrm.insert(nrm.end(), m.positions.size(), 0.f);
            else nrm.insert(nrm.end(), m.normals.begin(), m.normals.end());
        }
        for (int v : m.indices) idx.push_back(v + vbase);
        for (int t = 0; t < rm.tri_count; ++t) tri_mesh.push_back((int32_t)mi);
        meshes.push_back(rm);
    }
    std::vector<RMaterial> mats;
    for (const auto& m : D.materials) {
        RMaterial r{};
        r.type = m.type;
        for (int k = 0; k < 3; ++k) {
            r.kd[k] = m.kd[k];
            r.ks[k] = m.ks[k];
            r.kr[k] = m.kr[k];
            r.kt[k] = m.kt[k];
        }
        r.alpha_u = m.alpha_u;
        r.alpha_v = m.alpha_v;
        r.eta = m.eta;
        r.mirror_kr = m.mirror_kr;
        r.kd_tex = m.kd_texture;
        for (int k = 0; k < 3; ++k) {  // Fresnel::createFromIOR (BSDFs/Fresnel.h:27-31), host float
            float t = (m.eta - 1.f) / (m.eta + 1.f);
            r.f0[k] = m.has_f0 ? m.f0[k] : t * t;  // metal: its complex-IOR (or copper) f0
        }
        mats.push_back(r);
    }
    std::vector<RLight> lights;
    for (const auto& l : D.lights) {
        RLight r{};
        for (int k = 0; k < 3; ++k) r.L[k] = l.L[k];
        r.mesh = l.mesh;
        r.kind = l.kind == 1 ? kLightEnvironment : kLightArea;
        r.tex = l.texture;
        for (int row = 0; row < 3; ++row)  // glm::mat3(worldToLight): the upper-left 3x3
            for (int c = 0; c < 3; ++c) r.w2l[row * 3 + c] = l.world_to_light[c * 4 + row];
        lights.push_back(r);
    }
    // per-vertex texture coordinates, zero for meshes without them
    std::vector<float> uv;
    bool any_uv = false;
    for (const auto& m : D.meshes) any_uv |= !m.uvs.empty();
    if (any_uv)
        for (const auto& m : D.meshes) {
            if (m.uvs.empty()) uv.insert(uv.end(), m.positions.size() / 3 * 2, 0.f);
            else uv.insert(uv.end(), m.uvs.begin(), m.uvs.end());
        }
    sc->n_tri = (int64_t)idx.size() / 3;
    sc->n_vert = (int64_t)pos.size() / 3;
    cav_status st = CAV_OK;
    if ((st = upload((void**)&sc->d_pos, pos.data(), pos.size() * 4)) ||
        (st = upload((void**)&sc->d_idx, idx.data(), idx.size() * 4)) ||
        (st = upload((void**)&sc->d_tri_mesh, tri_mesh.data(), tri_mesh.size() * 4)) ||
        (st = upload((void**)&sc->d_meshes, meshes.data(), meshes.size() * sizeof(RMesh))) ||
        (st = upload((void**)&sc->d_mats, mats.data(), mats.size() * sizeof(RMaterial))) ||
        (st = upload((void**)&sc->d_lights, lights.data(), lights.size() * sizeof(RLight))) ||
        (st = ctx_halton(ctx, sc))) {
        scene_release(sc, stream, async);
        return st;
    }
    if ((any_normals && (st = upload((void**)&sc->d_nrm, nrm.data(), nrm.size() * 4))) ||
        (any_uv && (st = upload((void**)&sc->d_uv, uv.data(), uv.size() * 4)))) {
        scene_release(sc, stream, async);
        return st;
    }
    // image textures as the reference creates them (Core/Texture.h allocate): uchar4 texels
    // read as normalized floats (8-bit images) or float4 texels read as they are (OpenEXR),
    // bilinear filtering, wrapped normalized coordinates
    for (const auto& t : D.textures) {
        cudaChannelFormatDesc fmt = t.is_float ? cudaCreateChannelDesc<float4>() : cudaCreateChannelDesc<uchar4>();
        cudaArray_t arr = nullptr;
        if (cudaMallocArray(&arr, &fmt, t.width, t.height) != cudaSuccess) {
            cudaGetLastError();
            scene_release(sc, stream, async);
            return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "texture allocation failed");
        }
        sc->tex_arrays.push_back(arr);
        const size_t texel = t.is_float ? sizeof(float4) : 4;
        cudaMemcpy2DToArray(arr, 0, 0, t.is_float ? (const void*)t.rgbaf.data() : (const void*)t.rgba.data(),
                            texel * t.width, texel * t.width, t.height, cudaMemcpyHostToDevice);
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = cudaAddressModeWrap;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = t.is_float ? cudaReadModeElementType : cudaReadModeNormalizedFloat;
        td.normalizedCoords = 1;
        cudaTextureObject_t obj = 0;
        if (cudaCreateTextureObject(&obj, &res, &td, nullptr) != cudaSuccess) {
            cudaGetLastError();
            scene_release(sc, stream, async);
            return set_error(ctx, CAV_ERR_CUDA, "texture object creation failed");
        }
        sc->tex_objects.push_back(obj);
    }
    if (!sc->tex_objects.empty() &&
        (st = upload((void**)&sc->d_tex, sc->tex_objects.data(), sc->tex_objects.size() * sizeof(cudaTextureObject_t)))) {
        scene_release(sc, stream, async);
        return st;
    }
    *out = sc;
    return CAV_OK;
}

// Releases a scene and its tree.  async: stream-ordered frees on `s` (scenes uploaded with
// async = true); the Halton tables belong to the context.
void scene_release(cav_scene* sc, cudaStream_t s, bool async) {
    if (!sc) return;
    bvh_release(sc->bvh, s, async);
    void* arrays[] = {sc->d_pos, sc->d_idx, sc->d_nrm, sc->d_tri_mesh, sc->d_meshes, sc->d_mats,
                      sc->d_lights, sc->d_uv, sc->d_tex};
    for (void* p : arrays) {
        if (!p) continue;
        if (async) cudaFreeAsync(p, s);
        else cudaFree(p);
    }
    for (cudaTextureObject_t t : sc->tex_objects) cudaDestroyTextureObject(t);
    for (cudaArray_t a : sc->tex_arrays) cudaFreeArray(a);
    if (sc->graph_stream) {
        cudaStreamSynchronize(sc->graph_stream);
        cudaStreamDestroy(sc->graph_stream);
    }
    for (cudaEvent_t e : sc->log.pool) cudaEventDestroy(e);
    if (sc->log.totals_h) cudaFreeHost(sc->log.totals_h);
    delete sc;
}

void scene_geometry(const cav_scene* sc, const float** pos, int64_t* nv, const int32_t** idx, const int32_t** mesh,
                    int64_t* nt) {
    *pos = sc->d_pos;
    *nv = sc->n_vert;
    *idx = sc->d_idx;
    *mesh = sc->d_tri_mesh;
    *nt = sc->n_tri;
}

void scene_set_bvh(cav_scene* sc, cav_bvh* bvh, int rounds) {
    sc->bvh = bvh;
    sc->bvh_rounds = rounds;
}

int scene_spp(const cav_scene* sc) { return sc->desc.spp; }

// Parse result -> uploaded scene with its BVH, synchronously (cav_scene_load_pbrt).
cav_status scene_from_desc(cav_ctx* ctx, cavpbrt::Scene&& desc, int bvh_rounds, cav_scene** out) {
    cav_scene* sc = nullptr;
    cav_status st = scene_upload(ctx, std::move(desc), nullptr, false, &sc);
    if (st != CAV_OK) return st;
    const cavpbrt::Scene& D = sc->desc;
    // BVH over the global triangle list; rounds -1 = the reference's default
    // (3, or 10 when spp >= 64; Core/Scene.cu:141-146)
    if (bvh_rounds < 0) bvh_rounds = D.spp >= 64 ? 10 : 3;
    sc->bvh_rounds = bvh_rounds;
    st = build_bvh(ctx, sc->d_pos, sc->n_vert, sc->d_idx, sc->d_tri_mesh, sc->n_tri, nullptr, bvh_rounds, nullptr,
                   &sc->bvh);
    if (st != CAV_OK) {
        scene_release(sc, nullptr, false);
        return st;
    }
    CAV_CUDA(ctx, cudaDeviceSynchronize());
    *out = sc;
    return CAV_OK;
}

// Optional capture of one bounce's extend-stage rays (first chunk only), for timing other
// traversal implementations on exactly the rays the renderer traces.
struct RayCapture {
    int depth = -1;
    cav_ray* out = nullptr;
    int64_t capacity = 0;
    int64_t* count = nullptr;
};

cav_status render_path(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                       cudaStream_t s, const RayCapture* cap = nullptr, bool direct = false) {
    const cavpbrt::Scene& D = sc->desc;
    int W, H;
    film_size(sc, opts, W, H);
    const int spp = opts && opts->spp > 0 ? opts->spp : D.spp;
    const int max_depth = direct ? 1 : (opts && opts->max_depth > 0 ? opts->max_depth : D.max_depth);
    const int64_t pixels = (int64_t)W * H;
    const int64_t total = pixels * spp;
    // the camera samples of this render: all, or one shard [sample_begin, sample_end)
    const int64_t s_begin = opts && opts->sample_begin > 0 ? opts->sample_begin : 0;
    const int64_t s_end = opts && opts->sample_end > 0 ? std::min(opts->sample_end, total) : total;
    if (s_begin > s_end) return set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "sample_begin after sample_end");
    if (s_begin == s_end) return CAV_OK;
    int64_t chunk = opts && opts->max_paths_in_flight > 0 ? opts->max_paths_in_flight : (int64_t)1 << 22;
    chunk = std::min(chunk, s_end - s_begin);
    // path state + queues for `chunk` paths
    size_t need = 0;
    auto acc = [&](size_t bytes) { need += bytes + 256; };
    acc(8 * chunk); acc(8 * chunk); acc(12 * chunk); acc(12 * chunk); acc(4 * chunk); acc(chunk);
    acc(4 * chunk); acc(32 * chunk); acc(4 * chunk); acc(32 * chunk);
    acc(4 * chunk); acc(4 * chunk); acc(8 * chunk);
    acc(32 * chunk); acc(4 * chunk); acc(8 * chunk); acc(4 * chunk); acc(12 * chunk); acc(chunk); acc(64);
    void* base = nullptr;
    CAV_CUDA(ctx, dev_alloc(ctx, &base, need, s, true));
    struct FreeAsync {  // path state is released on every exit path, stream-ordered
        void* p;
        cudaStream_t s;
        ~FreeAsync() { cudaFreeAsync(p, s); }
    } free_base{base, s};
    unsigned char* p = (unsigned char*)base;
    Paths P;
    P.sample_index = carve<uint64_t>(p, chunk);
    P.film_xy = carve<float2>(p, chunk);
    P.result = carve<float>(p, 3 * chunk);
    P.throughput = carve<float>(p, 3 * chunk);
    P.mat_pdf = carve<float>(p, chunk);
    P.delta = carve<uint8_t>(p, chunk);
    Queues Q;
    Q.active = carve<int32_t>(p, chunk);
    Q.rays = carve<cav_ray>(p, chunk);
    Q.next_active = carve<int32_t>(p, chunk);
    Q.next_rays = carve<cav_ray>(p, chunk);
    Q.hit_prim = carve<int32_t>(p, chunk);
    Q.hit_t = carve<float>(p, chunk);
    Q.hit_uv = carve<float>(p, 2 * chunk);
    Q.shadow_rays = carve<cav_ray>(p, chunk);
    Q.shadow_limit = carve<float>(p, chunk);
    Q.shadow_excl = carve<int32_t>(p, 2 * chunk);
    Q.shadow_path = carve<int32_t>(p, chunk);
    Q.shadow_contrib = carve<float>(p, 3 * chunk);
    Q.shadow_occ = carve<uint8_t>(p, chunk);
    Q.counters = carve<uint32_t>(p, 16);

    DevScene S = dev_scene_of(sc);
    S.direct = direct ? 1 : 0;
    Camera cam = camera_of(sc, W, H);
    const uint32_t tflags = opts && (opts->flags & CAV_RENDER_FAST_TRACE) ? CAV_TRACE_FAST : CAV_TRACE_EXACT;
    uint32_t counts[2];
    auto& log = sc->log;
    log.reset();
    log.start = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.start, s));
    log.paths = s_end - s_begin;
    if (cap && cap->count) *cap->count = 0;
    for (int64_t first = s_begin; first < s_end; first += chunk) {
        const int64_t m = std::min(chunk, s_end - first);
        k_generate<<<div_up(m, kThreads), kThreads, 0, s>>>(cam, S.halton, spp, first, m, P, Q);
        int64_t n = m;
        // genCameraSampleSPPs stores the sampling state in the CameraSample BEFORE drawing the
        // two jitter dimensions from its local copy (Core/Sampler.cu:43-47), so a path's
        // first bounce starts again at dimension 0.
        int dim0 = 0;
        for (int depth = 0; n > 0 && depth < max_depth; ++depth) {
            if (cap && first == s_begin && depth == cap->depth && cap->out) {
                const int64_t k = std::min(n, cap->capacity);
                CAV_CUDA(ctx, cudaMemcpyAsync(cap->out, Q.rays, sizeof(cav_ray) * k, cudaMemcpyDeviceToDevice, s));
                if (cap->count) *cap->count = k;
            }
            cudaEvent_t e0 = log.next(), e1 = log.next(), e2 = log.next();
            CAV_CUDA(ctx, cudaEventRecord(e0, s));
            cav_status st = trace_closest(ctx, sc->bvh, Q.rays, n, Q.hit_prim, Q.hit_t, Q.hit_uv, tflags, s,
                                          ctx->d_counters + 6);
            if (st != CAV_OK) return st;
            CAV_CUDA(ctx, cudaEventRecord(e1, s));
            CAV_CUDA(ctx, cudaMemsetAsync(Q.counters, 0, 8, s));
            k_shade<<<div_up(n, kThreads), kThreads, 0, s>>>(S, depth, dim0, n, P, Q);
            CAV_CUDA(ctx, cudaEventRecord(e2, s));
            CAV_CUDA(ctx, cudaMemcpyAsync(counts, Q.counters, 8, cudaMemcpyDeviceToHost, s));
            CAV_CUDA(ctx, cudaStreamSynchronize(s));
            log.closest.emplace_back(e0, e1);
            log.shade.emplace_back(e1, e2);
            log.closest_rays += n;
            log.shadow_rays += counts[1];
            log.bounces = std::max(log.bounces, depth + 1);
            if (counts[1] > 0) {
                cudaEvent_t e3 = log.next(), e4 = log.next();
                CAV_CUDA(ctx, cudaEventRecord(e3, s));
                st = trace_any(ctx, sc->bvh, Q.shadow_rays, Q.shadow_limit, Q.shadow_excl, counts[1], Q.shadow_occ,
                               tflags, s, ctx->d_counters + 7);
                if (st != CAV_OK) return st;
                CAV_CUDA(ctx, cudaEventRecord(e4, s));
                log.any.emplace_back(e3, e4);
                k_add_direct<<<div_up(counts[1], kThreads), kThreads, 0, s>>>(counts[1], P, Q);
            }
            std::swap(Q.active, Q.next_active);
            std::swap(Q.rays, Q.next_rays);
            n = counts[0];
            dim0 += S.cont_dim + 2 + (depth > 3 ? 1 : 0);
        }
        k_film<<<div_up(m, kThreads), kThreads, 0, s>>>(m, P, W, H, D.filter_xwidth, D.filter_ywidth,
                                                         d_sum, d_wsum);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    log.end = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.end, s));
    return CAV_OK;
}

// ------------------------------------------------------------------ graph-replayed render
// The path integrator with every queue size kept on the device: the traversal kernels read
// their ray counts from the counters the previous kernel wrote, shading kernels run over the
// chunk capacity and stop at the device count.  One chunk's whole chain (generate, max_depth
// x (extend, shade, shadow, accumulate), film) is captured once as a CUDA graph and replayed
// for every chunk; the chunk's sample range comes from a device table indexed by a device
// counter that the graph's last node advances.  Bounces past the last live path launch
// kernels that exit at once.
namespace {
__global__ void k_chunk_begin(const int64_t* table, const int32_t* idx, int64_t* fc, uint32_t* cnt, int nslots) {
    const int i = *idx;
    fc[0] = table[2 * i];
    fc[1] = table[2 * i + 1];
    for (int k = 0; k < nslots; ++k) cnt[k] = 0;
    cnt[nslots] = (uint32_t)table[2 * i + 1];  // the extend queue size of bounce 0
}

__global__ void k_chunk_end(int32_t* idx, const uint32_t* cnt, int max_depth, unsigned long long* totals) {
    *idx += 1;
    unsigned long long closest = cnt[2 * max_depth], shadow = 0;
    for (int d = 0; d < max_depth; ++d) {
        if (d + 1 < max_depth) closest += cnt[2 * d];
        shadow += cnt[2 * d + 1];
    }
    totals[0] += closest;
    totals[1] += shadow;
}

}  // namespace

cav_status render_path_graph(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                             cudaStream_t s, unsigned long long* counters) {
    // the traversals' work counters: the caller's (two words), else the context's
    if (!counters) counters = ctx->d_counters + 6;
    const cavpbrt::Scene& D = sc->desc;
    int W, H;
    film_size(sc, opts, W, H);
    const int spp = opts && opts->spp > 0 ? opts->spp : D.spp;
    const int max_depth = opts && opts->max_depth > 0 ? opts->max_depth : D.max_depth;
    const int64_t total = (int64_t)W * H * spp;
    int64_t chunk = opts && opts->max_paths_in_flight > 0 ? opts->max_paths_in_flight : (int64_t)1 << 22;
    chunk = std::min(chunk, total);
    const int64_t nchunks = (total + chunk - 1) / chunk;
    size_t need = 0;
    {
        auto acc = [&](size_t bytes) { need += bytes + 256; };
        acc(8 * chunk); acc(8 * chunk); acc(12 * chunk); acc(12 * chunk); acc(4 * chunk); acc(chunk);
        acc(4 * chunk); acc(32 * chunk); acc(4 * chunk); acc(32 * chunk);
        acc(4 * chunk); acc(4 * chunk); acc(8 * chunk);
        acc(32 * chunk); acc(4 * chunk); acc(8 * chunk); acc(4 * chunk); acc(12 * chunk); acc(chunk); acc(64);
        acc(16 * nchunks); acc(16); acc(4); acc(4 * (2 * max_depth + 2)); acc(16);
    }
    void* base = nullptr;
    CAV_CUDA(ctx, dev_alloc(ctx, &base, need, s, true));
    struct FreeAsync {
        void* p;
        cudaStream_t s;
        ~FreeAsync() { cudaFreeAsync(p, s); }
    } free_base{base, s};
    unsigned char* p = (unsigned char*)base;
    Paths P;
    P.sample_index = carve<uint64_t>(p, chunk);
    P.film_xy = carve<float2>(p, chunk);
    P.result = carve<float>(p, 3 * chunk);
    P.throughput = carve<float>(p, 3 * chunk);
    P.mat_pdf = carve<float>(p, chunk);
    P.delta = carve<uint8_t>(p, chunk);
    Queues Q0;
    Q0.active = carve<int32_t>(p, chunk);
    Q0.rays = carve<cav_ray>(p, chunk);
    Q0.next_active = carve<int32_t>(p, chunk);
    Q0.next_rays = carve<cav_ray>(p, chunk);
    Q0.hit_prim = carve<int32_t>(p, chunk);
    Q0.hit_t = carve<float>(p, chunk);
    Q0.hit_uv = carve<float>(p, 2 * chunk);
    Q0.shadow_rays = carve<cav_ray>(p, chunk);
    Q0.shadow_limit = carve<float>(p, chunk);
    Q0.shadow_excl = carve<int32_t>(p, 2 * chunk);
    Q0.shadow_path = carve<int32_t>(p, chunk);
    Q0.shadow_contrib = carve<float>(p, 3 * chunk);
    Q0.shadow_occ = carve<uint8_t>(p, chunk);
    Q0.counters = carve<uint32_t>(p, 16);
    int64_t* d_table = carve<int64_t>(p, 2 * nchunks);
    int64_t* d_fc = carve<int64_t>(p, 2);
    int32_t* d_idx = carve<int32_t>(p, 1);
    uint32_t* cnt = carve<uint32_t>(p, 2 * max_depth + 2);  // [2d] next rays, [2d+1] shadow rays, [2D] bounce-0 size
    unsigned long long* totals = carve<unsigned long long>(p, 2);
    std::vector<int64_t> table(2 * nchunks);
    for (int64_t c = 0; c < nchunks; ++c) {
        table[2 * c] = c * chunk;
        table[2 * c + 1] = std::min(chunk, total - c * chunk);
    }
    auto& log = sc->log;
    log.reset();
    log.start = log.next();
    log.paths = total;
    CAV_CUDA(ctx, cudaMemcpyAsync(d_table, table.data(), sizeof(int64_t) * 2 * nchunks, cudaMemcpyHostToDevice, s));
    CAV_CUDA(ctx, cudaMemsetAsync(d_idx, 0, 4, s));
    CAV_CUDA(ctx, cudaMemsetAsync(totals, 0, 16, s));
    CAV_CUDA(ctx, cudaStreamSynchronize(s));  // the table copy reads pageable host memory
    const DevScene S = dev_scene_of(sc);
    const Camera cam = camera_of(sc, W, H);
    const unsigned blocks = (unsigned)div_up(chunk, kThreads);
    const bool fast = opts && (opts->flags & CAV_RENDER_FAST_TRACE);
    if (fast) {  // the 8-wide view is built (with host checks) before the capture begins
        cav_status wst = ensure_wide(ctx, sc->bvh, s);
        if (wst != CAV_OK) return wst;
    }
    // capture and replay on the scene's own non-blocking stream (the legacy default stream
    // cannot be captured), ordered after and before the caller's stream by events
    const cudaStream_t caller = s;
    if (!sc->graph_stream) CAV_CUDA(ctx, cudaStreamCreateWithFlags(&sc->graph_stream, cudaStreamNonBlocking));
    s = sc->graph_stream;
    {
        cudaEvent_t fork = log.next();
        CAV_CUDA(ctx, cudaEventRecord(fork, caller));
        CAV_CUDA(ctx, cudaStreamWaitEvent(s, fork, 0));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CAV_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cav_status st = CAV_OK;
    {
        k_chunk_begin<<<1, 1, 0, s>>>(d_table, d_idx, d_fc, cnt, 2 * max_depth);
        k_generate<<<blocks, kThreads, 0, s>>>(cam, S.halton, spp, 0, 0, P, Q0, d_fc);
        Queues Q = Q0;
        int dim0 = 0;
        for (int depth = 0; depth < max_depth && st == CAV_OK; ++depth) {
            const uint32_t* n_dev = depth == 0 ? cnt + 2 * max_depth : cnt + 2 * (depth - 1);
            Q.counters = cnt + 2 * depth;
            st = fast ? trace_wide_closest(ctx, sc->bvh, Q.rays, INT64_MAX, n_dev, Q.hit_prim, Q.hit_t, Q.hit_uv, s,
                                           counters)
                      : trace_closest_dev(ctx, sc->bvh, Q.rays, n_dev, Q.hit_prim, Q.hit_t, Q.hit_uv, s,
                                          counters);
            if (st != CAV_OK) break;
            k_shade<<<blocks, kThreads, 0, s>>>(S, depth, dim0, 0, P, Q, n_dev);
            st = fast ? trace_wide_any(ctx, sc->bvh, Q.shadow_rays, Q.shadow_limit, Q.shadow_excl, INT64_MAX,
                                       cnt + 2 * depth + 1, Q.shadow_occ, s, counters + 1)
                      : trace_any_dev(ctx, sc->bvh, Q.shadow_rays, Q.shadow_limit, Q.shadow_excl, cnt + 2 * depth + 1,
                                      Q.shadow_occ, s, counters + 1);
            if (st != CAV_OK) break;
            k_add_direct<<<blocks, kThreads, 0, s>>>(0, P, Q, cnt + 2 * depth + 1);
            std::swap(Q.active, Q.next_active);
            std::swap(Q.rays, Q.next_rays);
            dim0 += S.cont_dim + 2 + (depth > 3 ? 1 : 0);
        }
        k_film<<<blocks, kThreads, 0, s>>>(0, P, W, H, D.filter_xwidth, D.filter_ywidth, d_sum, d_wsum, d_fc);
        k_chunk_end<<<1, 1, 0, s>>>(d_idx, cnt, max_depth, totals);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st != CAV_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    CAV_CUDA(ctx, ce);
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CAV_CUDA(ctx, ce);
    CAV_CUDA(ctx, cudaEventRecord(log.start, s));
    for (int64_t c = 0; c < nchunks; ++c) {
        ce = cudaGraphLaunch(exec, s);
        if (ce != cudaSuccess) break;
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(sc->log_totals_host(), totals, 16, cudaMemcpyDeviceToHost, s);
    cudaGraphExecDestroy(exec);  // released once the launches complete
    CAV_CUDA(ctx, ce);
    log.end = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.end, s));
    CAV_CUDA(ctx, cudaStreamWaitEvent(caller, log.end, 0));  // join: the film is ready on the caller's stream
    log.graph = true;
    return CAV_OK;
}

// ------------------------------------------------------------------ resumable render job
// The path integrator as a state machine advanced one bounce at a time by the serving loop
// (serve.cu), whose traversal launches merge the wavefronts of every live job.  Per chunk
// and bounce it launches exactly the kernels render_path launches, in the same order.
struct PathJob {
    cav_ctx* ctx = nullptr;
    cav_scene* sc = nullptr;
    int W = 0, H = 0;
    int spp = 0, max_depth = 0;
    int64_t total = 0, chunk = 0, first = 0, m = 0, n = 0;
    int64_t slice = 0;  // paths started per chunk (<= chunk, the state's capacity); 0: chunk
    int depth = 0, dim0 = 0;
    void* base = nullptr;
    float* d_sum = nullptr;
    float* d_wsum = nullptr;
    uint32_t* h_counts = nullptr;  // pinned: next rays, shadow rays
    Paths P;
    Queues Q;
    DevScene S;
    Camera cam;
    bool done = false;
};

static size_t path_state_bytes(int64_t chunk) {
    size_t need = 0;
    auto acc = [&](size_t bytes) { need += bytes + 256; };
    acc(8 * chunk); acc(8 * chunk); acc(12 * chunk); acc(12 * chunk); acc(4 * chunk); acc(chunk);
    acc(4 * chunk); acc(32 * chunk); acc(4 * chunk); acc(32 * chunk);
    acc(4 * chunk); acc(4 * chunk); acc(8 * chunk);
    acc(32 * chunk); acc(4 * chunk); acc(8 * chunk); acc(4 * chunk); acc(12 * chunk); acc(chunk); acc(64);
    return need;
}

static void job_chunk_sizes(const cav_scene* sc, const cav_render_opts* opts, int& spp, int& depth, int64_t& total,
                            int64_t& chunk) {
    const cavpbrt::Scene& D = sc->desc;
    int W, H;
    film_size(sc, opts, W, H);
    spp = opts && opts->spp > 0 ? opts->spp : D.spp;
    depth = opts && opts->max_depth > 0 ? opts->max_depth : D.max_depth;
    total = (int64_t)W * H * spp;
    chunk = opts && opts->max_paths_in_flight > 0 ? opts->max_paths_in_flight : (int64_t)1 << 22;
    chunk = std::min(chunk, total);
}

size_t render_state_bytes(int W, int H, int spp, int64_t max_paths) {
    const int64_t total = (int64_t)W * H * spp;
    const int64_t chunk = std::min<int64_t>(max_paths > 0 ? max_paths : (int64_t)1 << 22, total);
    return path_state_bytes(chunk) + sizeof(float) * 4 * (int64_t)W * H + 512;
}

size_t path_job_bytes(const cav_scene* sc, const cav_render_opts* opts) {
    int spp, depth;
    int64_t total, chunk;
    job_chunk_sizes(sc, opts, spp, depth, total, chunk);
    int W, H;
    film_size(sc, opts, W, H);
    return path_state_bytes(chunk) + sizeof(float) * 4 * (int64_t)W * H + 512;
}

cav_status path_job_create(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, int64_t slice, cudaStream_t s,
                           PathJob** out) {
    auto* J = new PathJob();
    J->ctx = ctx;
    J->sc = sc;
    job_chunk_sizes(sc, opts, J->spp, J->max_depth, J->total, J->chunk);
    film_size(sc, opts, J->W, J->H);
    const int64_t pixels = (int64_t)J->W * J->H;
    const size_t bytes = path_job_bytes(sc, opts);
    if (dev_alloc(ctx, &J->base, bytes, s, true) != cudaSuccess || cudaMallocHost(&J->h_counts, 16) != cudaSuccess) {
        cudaGetLastError();
        if (J->base) cudaFreeAsync(J->base, s);
        delete J;
        return set_error(ctx, CAV_ERR_OUT_OF_MEMORY, "render job: device allocation failed");
    }
    unsigned char* p = (unsigned char*)J->base;
    J->d_sum = carve<float>(p, 3 * pixels);
    J->d_wsum = carve<float>(p, pixels);
    const int64_t c = J->chunk;
    J->P.sample_index = carve<uint64_t>(p, c);
    J->P.film_xy = carve<float2>(p, c);
    J->P.result = carve<float>(p, 3 * c);
    J->P.throughput = carve<float>(p, 3 * c);
    J->P.mat_pdf = carve<float>(p, c);
    J->P.delta = carve<uint8_t>(p, c);
    J->Q.active = carve<int32_t>(p, c);
    J->Q.rays = carve<cav_ray>(p, c);
    J->Q.next_active = carve<int32_t>(p, c);
    J->Q.next_rays = carve<cav_ray>(p, c);
    J->Q.hit_prim = carve<int32_t>(p, c);
    J->Q.hit_t = carve<float>(p, c);
    J->Q.hit_uv = carve<float>(p, 2 * c);
    J->Q.shadow_rays = carve<cav_ray>(p, c);
    J->Q.shadow_limit = carve<float>(p, c);
    J->Q.shadow_excl = carve<int32_t>(p, 2 * c);
    J->Q.shadow_path = carve<int32_t>(p, c);
    J->Q.shadow_contrib = carve<float>(p, 3 * c);
    J->Q.shadow_occ = carve<uint8_t>(p, c);
    J->Q.counters = carve<uint32_t>(p, 16);
    J->S = dev_scene_of(sc);
    J->cam = camera_of(sc, J->W, J->H);
    CAV_CUDA(ctx, cudaMemsetAsync(J->d_sum, 0, sizeof(float) * 4 * pixels, s));
    J->first = 0;
    J->slice = slice > 0 ? std::min(slice, J->chunk) : J->chunk;
    J->m = std::min(J->slice, J->total);
    k_generate<<<div_up(J->m, kThreads), kThreads, 0, s>>>(J->cam, J->S.halton, J->spp, 0, J->m, J->P, J->Q);
    J->n = J->m;
    J->depth = 0;
    J->dim0 = 0;
    CAV_CUDA(ctx, cudaGetLastError());
    *out = J;
    return CAV_OK;
}

// The extend segment of the current bounce (0 rays when the job has none this tick).
int64_t path_job_extend(PathJob* J, TraceSeg* seg) {
    if (J->done || J->n <= 0) return 0;
    const cav_bvh* b = J->sc->bvh;
    *seg = TraceSeg{};
    seg->nodes = b->tnodes;
    seg->tris = b->tris;
    seg->cnodes = b->cnodes;  // set once the fast-mode view exists (ensure_wide)
    seg->ctris = b->ctris;
    seg->root_box = b->d_root_box;
    seg->rays = J->Q.rays;
    seg->prim = J->Q.hit_prim;
    seg->t = J->Q.hit_t;
    seg->uv = J->Q.hit_uv;
    return J->n;
}

cav_status path_job_shade(PathJob* J, cudaStream_t s) {
    cav_ctx* ctx = J->ctx;
    CAV_CUDA(ctx, cudaMemsetAsync(J->Q.counters, 0, 8, s));
    k_shade<<<div_up(J->n, kThreads), kThreads, 0, s>>>(J->S, J->depth, J->dim0, J->n, J->P, J->Q);
    CAV_CUDA(ctx, cudaMemcpyAsync(J->h_counts, J->Q.counters, 8, cudaMemcpyDeviceToHost, s));
    return CAV_OK;
}

// After the stream has caught up with path_job_shade: the shadow segment.
int64_t path_job_shadow(PathJob* J, TraceSeg* seg) {
    const int64_t k = J->h_counts[1];
    if (k <= 0) return 0;
    const cav_bvh* b = J->sc->bvh;
    *seg = TraceSeg{};
    seg->nodes = b->tnodes;
    seg->tris = b->tris;
    seg->cnodes = b->cnodes;  // set once the fast-mode view exists (ensure_wide)
    seg->ctris = b->ctris;
    seg->root_box = b->d_root_box;
    seg->rays = J->Q.shadow_rays;
    seg->limit = J->Q.shadow_limit;
    seg->excl = J->Q.shadow_excl;
    seg->occ = J->Q.shadow_occ;
    return k;
}

// Adds the unoccluded light samples, advances to the next bounce or chunk; returns whether
// the job has finished (its film complete on the stream).
cav_status path_job_advance(PathJob* J, cudaStream_t s, bool* finished) {
    cav_ctx* ctx = J->ctx;
    const int64_t k = J->h_counts[1];
    if (k > 0) k_add_direct<<<div_up(k, kThreads), kThreads, 0, s>>>(k, J->P, J->Q);
    std::swap(J->Q.active, J->Q.next_active);
    std::swap(J->Q.rays, J->Q.next_rays);
    J->n = J->h_counts[0];
    J->dim0 += J->S.cont_dim + 2 + (J->depth > 3 ? 1 : 0);
    J->depth += 1;
    if (J->n <= 0 || J->depth >= J->max_depth) {
        const cavpbrt::Scene& D = J->sc->desc;
        k_film<<<div_up(J->m, kThreads), kThreads, 0, s>>>(J->m, J->P, J->W, J->H, D.filter_xwidth,
                                                            D.filter_ywidth, J->d_sum, J->d_wsum);
        J->first += J->m;
        if (J->first < J->total) {
            J->m = std::min(J->slice, J->total - J->first);
            k_generate<<<div_up(J->m, kThreads), kThreads, 0, s>>>(J->cam, J->S.halton, J->spp, J->first, J->m, J->P,
                                                                  J->Q);
            J->n = J->m;
            J->depth = 0;
            J->dim0 = 0;
        } else {
            J->done = true;
            J->n = 0;
        }
    }
    CAV_CUDA(ctx, cudaGetLastError());
    *finished = J->done;
    return CAV_OK;
}

// The paths the job's next chunk starts (clamped to the state's capacity).
void path_job_set_slice(PathJob* J, int64_t slice) { J->slice = slice > 0 ? std::min(slice, J->chunk) : J->chunk; }

int64_t path_job_capacity(const PathJob* J) { return J->chunk; }

void path_job_film(PathJob* J, float** sum, float** wsum, int64_t* pixels) {
    *sum = J->d_sum;
    *wsum = J->d_wsum;
    *pixels = (int64_t)J->W * J->H;
}

void path_job_destroy(PathJob* J, cudaStream_t s) {
    if (!J) return;
    if (J->base) cudaFreeAsync(J->base, s);
    if (J->h_counts) cudaFreeHost(J->h_counts);
    delete J;
}

}  // namespace cav

// ======================================================================== C ABI
extern "C" {

cav_status cav_scene_load_pbrt(cav_ctx* ctx, const char* path, int spp_override, const char* integrator_override,
                               int bvh_rounds, cav_scene** out) {
    if (!ctx || !path || !out) return CAV_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    cavpbrt::Overrides ov;
    ov.spp = spp_override;
    if (integrator_override) ov.integrator = integrator_override;
    cavpbrt::Scene desc;
    try {
        desc = cavpbrt::load_file(path, ov);
    } catch (const std::exception& e) {
        return cav::set_error(ctx, CAV_ERR_INVALID_ARGUMENT, std::string("pbrt: ") + e.what());
    }
    return cav::scene_from_desc(ctx, std::move(desc), bvh_rounds, out);
}

cav_status cav_scene_free(cav_scene* sc) {
    if (!sc) return CAV_OK;
    cudaSetDevice(sc->device);
    cav::scene_release(sc, nullptr, false);
    return CAV_OK;
}

cav_status cav_scene_info(const cav_scene* sc, cav_scene_info_t* info) {
    if (!sc || !info) return CAV_ERR_INVALID_ARGUMENT;
    info->width = sc->desc.width;
    info->height = sc->desc.height;
    info->spp = sc->desc.spp;
    info->max_depth = sc->desc.max_depth;
    info->triangles = sc->n_tri;
    info->meshes = (int)sc->desc.meshes.size();
    info->lights = (int)sc->desc.lights.size();
    info->bvh_rounds = sc->bvh_rounds;
    info->integrator = sc->desc.integrator == "rlpath" ? 1 : (sc->desc.integrator == "directlighting" ? 3 : 0);
    return CAV_OK;
}

const cav_bvh* cav_scene_bvh(const cav_scene* sc) { return sc ? sc->bvh : nullptr; }

cav_status cav_render(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* film_sum, float* film_weight,
                      void* stream) {
    if (!ctx || !sc || !film_sum || !film_weight) return CAV_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    int W, H;
    cav::film_size(sc, opts, W, H);
    const int64_t pixels = (int64_t)W * H;
    CAV_CUDA(ctx, cudaMemsetAsync(film_sum, 0, sizeof(float) * 3 * pixels, s));
    CAV_CUDA(ctx, cudaMemsetAsync(film_weight, 0, sizeof(float) * pixels, s));
    // integrator: the options' choice when given (> 0 selects one), else the scene's
    int integrator = sc->desc.integrator == "rlpath" ? 1 : (sc->desc.integrator == "directlighting" ? 3 : 0);
    if (opts && opts->integrator > 0) integrator = opts->integrator;
    if (opts && opts->integrator < 0) integrator = 0;
    const bool ranged = opts && (opts->sample_begin > 0 || opts->sample_end > 0);
    if (ranged && (integrator == 1 || integrator == 2))
        return cav::set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "sample ranges are for the path and direct integrators");
    if (integrator == 1) return cav::render_rlpath(ctx, sc, opts, film_sum, film_weight, s);
    if (integrator == 2) return cav_render_guided(ctx, sc, opts, nullptr, nullptr, film_sum, film_weight, s, nullptr);
    if (integrator == 3) return cav::render_path(ctx, sc, opts, film_sum, film_weight, s, nullptr, true);
    if (integrator != 0) return cav::set_error(ctx, CAV_ERR_INVALID_ARGUMENT, "unknown integrator");
    if (opts && (opts->flags & CAV_RENDER_GRAPH) && !ranged)
        return cav::render_path_graph(ctx, sc, opts, film_sum, film_weight, s);
    return cav::render_path(ctx, sc, opts, film_sum, film_weight, s);
}

cav_status cav_render_stats(const cav_scene* sc, cav_render_stats_t* out) {
    if (!sc || !out) return CAV_ERR_INVALID_ARGUMENT;
    const auto& L = sc->log;
    *out = cav_render_stats_t{};
    out->paths = L.paths;
    out->closest_rays = L.closest_rays;
    out->shadow_rays = L.shadow_rays;
    out->bounces = L.bounces;
    if (!L.start || !L.end) return CAV_OK;
    if (cudaEventSynchronize(L.end) != cudaSuccess) return CAV_ERR_CUDA;
    if (L.graph && L.totals_h) {
        out->closest_rays = (int64_t)L.totals_h[0];
        out->shadow_rays = (int64_t)L.totals_h[1];
    }
    auto sum = [](const std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v) {
        double t = 0;
        for (const auto& p : v) {
            float ms = 0;
            cudaEventElapsedTime(&ms, p.first, p.second);
            t += ms;
        }
        return (float)t;
    };
    out->ms_closest = sum(L.closest);
    out->ms_shade = sum(L.shade);
    out->ms_any = sum(L.any);
    cudaEventElapsedTime(&out->ms_total, L.start, L.end);
    return CAV_OK;
}

cav_status cav_render_capture_rays(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, int depth,
                                   cav_ray* rays_out, int64_t capacity, int64_t* count) {
    if (!ctx || !sc || !rays_out || !count || depth < 0 || capacity <= 0) return CAV_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    int W, H;
    cav::film_size(sc, opts, W, H);
    const int64_t pixels = (int64_t)W * H;
    float* film = nullptr;
    CAV_CUDA(ctx, cudaMalloc(&film, sizeof(float) * 4 * pixels));
    cav_render_opts o = opts ? *opts : cav_render_opts{0, 0, 0, 0, 0, 0, 0};
    // one chunk is enough: the capture is taken from the first chunk
    const int spp = o.spp > 0 ? o.spp : sc->desc.spp;
    const int64_t total = pixels * spp;
    if (o.max_paths_in_flight <= 0) o.max_paths_in_flight = (int64_t)1 << 22;
    o.max_paths_in_flight = std::min(o.max_paths_in_flight, total);
    cav::RayCapture cap;
    cap.depth = depth;
    cap.out = rays_out;
    cap.capacity = capacity;
    cap.count = count;
    cudaMemset(film, 0, sizeof(float) * 4 * pixels);
    cav_status st = cav::render_path(ctx, sc, &o, film, film + 3 * pixels, nullptr, &cap);
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(film);
    if (st == CAV_OK && e != cudaSuccess) st = cav::cuda_error(ctx, e, "render capture");
    return st;
}

cav_status cav_render_to_host(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* host_sum,
                              float* host_weight, float* ms_out) {
    if (!ctx || !sc || !host_sum || !host_weight) return CAV_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    int W, H;
    cav::film_size(sc, opts, W, H);
    const int64_t pixels = (int64_t)W * H;
    float* d = nullptr;
    CAV_CUDA(ctx, cudaMalloc(&d, sizeof(float) * 4 * pixels));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, nullptr);
    cav_status st = cav_render(ctx, sc, opts, d, d + 3 * pixels, nullptr);
    cudaEventRecord(b, nullptr);
    if (st == CAV_OK) {
        cudaError_t e = cudaMemcpy(host_sum, d, sizeof(float) * 3 * pixels, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(host_weight, d + 3 * pixels, sizeof(float) * pixels, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cav::cuda_error(ctx, e, "cudaMemcpy film");
        if (ms_out) cudaEventElapsedTime(ms_out, a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    return st;
}

}  // extern "C"
