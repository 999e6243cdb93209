// MLP-guided path integrator: the plain path tracer whose continuation at non-delta
// surfaces is drawn, with probability alpha, from the learned vMF mixture of mlp.cu
// instead of the BSDF.  One-sample MIS over the two strategies: a direction drawn either way
// is weighted by the mixture density alpha q(w) + (1 - alpha) p_bsdf(w), which keeps the
// estimator unbiased for any network; light samples are MIS-weighted against that same
// density.  The render proceeds in passes (1, 1, 2, 4, ... spp); after each pass the network
// trains on the pass's path vertices: the direction taken and the luminance of the radiance
// that came back through it divided by the throughput at the vertex (the weight of the
// loss -w log q(w) that pulls q toward f |cos| L_i).  The first pass samples the BSDF only.
// Halton dimensions: 16 per bounce (light 0-7, roulette 8, BSDF 9-10, strategy 11,
// mixture 12-14).
#include <cstdio>
#include <cstring>

#include "render_common.cuh"

namespace cav {
namespace mlp_dev {
// the mixture maths of mlp.cu, restated for this translation unit
constexpr int kLobes = 8;
constexpr int kOut = 32;
constexpr float kPi = 3.14159265358979323846f;
struct Lobe {
    float w, mx, my, mz, kappa, norm;
};
__device__ inline float sig(float x) { return 1.f / (1.f + __expf(-x)); }
__device__ inline float softplus(float x) { return x > 15.f ? x : log1pf(__expf(x)); }
__device__ inline void decode(const float* o, Lobe (&L)[kLobes]) {
    float mx = -INFINITY;
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, o[4 * k]);
    float s = 0.f;
    for (int k = 0; k < kLobes; ++k) {
        L[k].w = __expf(o[4 * k] - mx);
        s += L[k].w;
    }
    for (int k = 0; k < kLobes; ++k) {
        L[k].w /= s;
        float st, ct, sp, cp;
        __sincosf(kPi * sig(o[4 * k + 1]), &st, &ct);
        __sincosf(2.f * kPi * sig(o[4 * k + 2]), &sp, &cp);
        L[k].mx = st * cp;
        L[k].my = st * sp;
        L[k].mz = ct;
        float kap = fminf(softplus(o[4 * k + 3]) + 0.01f, 500.f);
        L[k].kappa = kap;
        L[k].norm = kap / (2.f * kPi * (1.f - __expf(-2.f * kap)));
    }
}
__device__ inline float pdf(const Lobe (&L)[kLobes], f3 d) {
    float p = 0.f;
    for (int k = 0; k < kLobes; ++k)
        p += L[k].w * L[k].norm * __expf(L[k].kappa * (L[k].mx * d.x + L[k].my * d.y + L[k].mz * d.z - 1.f));
    return p;
}
__device__ inline f3 sample(const Lobe (&L)[kLobes], float u0, float u1, float u2) {
    int k = 0;
    float acc = L[0].w;
    while (k < kLobes - 1 && u0 >= acc) acc += L[++k].w;
    const float kap = L[k].kappa;
    float c = fminf(1.f, fmaxf(-1.f, 1.f + logf(u1 + (1.f - u1) * __expf(-2.f * kap)) / kap));
    float s = sqrtf(fmaxf(0.f, 1.f - c * c));
    float sp, cp;
    __sincosf(2.f * kPi * u2, &sp, &cp);
    f3 n = mk(L[k].mx, L[k].my, L[k].mz);
    f3 t = fabsf(n.x) < 0.5f ? mk(0.f, -n.z, n.y) : mk(n.z, 0.f, -n.x);
    t = normalize3(t);
    f3 b = cross3(n, t);
    return t * (s * cp) + b * (s * sp) + n * c;
}
}  // namespace mlp_dev

namespace {

constexpr int kDims = 16;

struct Records {  // per path and depth
    float* feat;     // 5
    float* dir;      // 3
    float* thr;      // 3
    float* res;      // 3: radiance of the path before its continuation from this vertex
    uint8_t* valid;
    int depth;       // max depth (record stride)
};

struct TrainBuf {
    float* feat;
    float* dir;
    float* w;
    uint32_t* count;
    uint32_t cap;
};

__device__ inline bool guidable(const Bsdf& B) { return !B.is_delta(); }

// Camera samples of one pass: this_spp samples per pixel, pixel-major, whose Halton indices
// continue after done_spp (the reference's sppBySpp rounds, Core/Sampler.cu:29-51).
__global__ void k_generate_pass(Camera cam, Halton H, int spp_total, int this_spp, int done_spp, int64_t first,
                                int64_t count, Paths P, Queues Q) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    int64_t s = first + i;
    int64_t pixel = s / this_spp;
    int x = (int)(pixel % cam.width), y = (int)(pixel / cam.width);
    uint64_t index = (uint64_t)pixel * spp_total + (uint64_t)done_spp + (uint64_t)(s % this_spp);
    int dim = 0;
    float sx = x + halton(H, index, dim);
    float sy = y + halton(H, index, dim);
    f3 pl = mk(sx - cam.width / 2.f, cam.height / 2.f - sy, cam.depth);
    f3 o = apply_pt(cam.c2w, mk(0, 0, 0));
    f3 d = normalize3(apply_pt(cam.c2w, pl) - o);
    P.sample_index[i] = index;
    P.film_xy[i] = make_float2(sx, sy);
    P.result[3 * i] = P.result[3 * i + 1] = P.result[3 * i + 2] = 0.f;
    P.throughput[3 * i] = P.throughput[3 * i + 1] = P.throughput[3 * i + 2] = 1.f;
    P.mat_pdf[i] = 1.f;
    P.delta[i] = 1;
    Q.active[i] = (int32_t)i;
    Q.rays[i] = cav_ray{o.x, o.y, o.z, 0.f, d.x, d.y, d.z, INFINITY};
}

// surface features: position in the scene box, normal angles, all in [0, 1]
__global__ void k_g_features(DevScene S, const float* box, int64_t n, Queues Q, float* feat) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float f[5] = {0, 0, 0, 0, 0};
    const int prim = Q.hit_prim[j];
    if (prim >= 0) {
        const cav_ray r = Q.rays[j];
        f3 pos = mk(r.ox, r.oy, r.oz) + Q.hit_t[j] * mk(r.dx, r.dy, r.dz);
        const RMesh& M = S.meshes[S.tri_mesh[prim]];
        f3 nrm = tri_normal(S, M, prim, Q.hit_uv[2 * j], Q.hit_uv[2 * j + 1]);
        for (int k = 0; k < 3; ++k) {
            float lo = box[k], hi = box[3 + k];
            float v = (k == 0 ? pos.x : k == 1 ? pos.y : pos.z);
            f[k] = hi > lo ? fminf(1.f, fmaxf(0.f, (v - lo) / (hi - lo))) : 0.5f;
        }
        f[3] = acosf(fminf(1.f, fmaxf(-1.f, nrm.z))) / mlp_dev::kPi;
        f[4] = (atan2f(nrm.y, nrm.x) + mlp_dev::kPi) / (2.f * mlp_dev::kPi);
    }
    for (int k = 0; k < 5; ++k) feat[j * 5 + k] = f[k];
}

// k_shade of the path integrator with the guided continuation and its MIS density.
// 2 blocks per SM (128 registers, about 200 bytes spilled) instead of 1 at 146 registers:
// the 640x360 64-spp guided render of the aperture scene took 163 ms at 1 block, 153 at 2
// and 152 at 3 (80 registers, about 1 KB spilled).
__global__ void __launch_bounds__(kThreads, 2) k_g_shade(DevScene S, int depth, int dim0, int64_t n, Paths P, Queues Q, const float* feat,
                          const float* mout, float alpha, Records R, int record) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
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
        f3 pos = ro + t * rd;
        f3 nrm = tri_normal(S, M, prim, u, v);
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
        const f3 wo = to_local(fr, rd * -1.f);
        const bool guided = alpha > 0.f && guidable(B);
        mlp_dev::Lobe Lb[mlp_dev::kLobes];
        if (guided) mlp_dev::decode(mout + j * mlp_dev::kOut, Lb);
        // continuation density of a world direction
        auto cont_pdf = [&](f3 dw, f3 dl) {
            float pb = B.pdf(dl, wo);
            return guided ? alpha * mlp_dev::pdf(Lb, dw) + (1.f - alpha) * pb : pb;
        };
        // ---- light sample
        int dim = dim0;
        int li = halton_int(S.halton, index, dim, S.n_lights);
        dim += 4;
        const LightSample ls = sample_light(S, S.lights[li], pos, index, dim);  // 2 or 3 of the 3 reserved
        const float light_pdf = ls.pdf;
        const f3 dir = ls.dir;
        const f3 incident = ls.incident;
        if (isfinite(light_pdf)) {
            f3 wi = to_local(fr, dir);
            float w = mis_power(light_pdf, cont_pdf(dir, wi));
            float cosine = fabsf(dot3(dir, nrm));
            f3 mult = thr * (float)S.n_lights / light_pdf;
            contrib = incident * B.eval(wi, wo) * cosine * mult * w;
            if (!all_zero(contrib)) {
                emit_shadow = true;
                shadow = cav_ray{pos.x, pos.y, pos.z, 0.f, dir.x, dir.y, dir.z, INFINITY};
                limit = ls.dist;
                excl = make_int2(mesh, ls.target);
            }
        }
        // ---- continuation
        bool alive = true;
        if (depth > 3) {
            dim = dim0 + 8;
            float q = 1;
            q = fminf(q, 1 - thr.x);
            q = fminf(q, 1 - thr.y);
            q = fminf(q, 1 - thr.z);
            q = fmaxf(q, 0.05f);
            if (halton(S.halton, index, dim) < q) alive = false;
            else thr = thr / (1.f - q);
        }
        if (alive) {
            f3 wi, nd, f;
            float p = 0.f;
            dim = dim0 + 11;
            const float usel = halton(S.halton, index, dim);
            if (guided && usel < alpha) {
                float u0 = halton(S.halton, index, dim);
                float u1 = halton(S.halton, index, dim);
                float u2 = halton(S.halton, index, dim);
                nd = mlp_dev::sample(Lb, u0, u1, u2);
                wi = to_local(fr, nd);
                f = B.eval(wi, wo);
            } else {
                dim = dim0 + 9;
                float u0 = halton(S.halton, index, dim);
                float u1 = halton(S.halton, index, dim);
                f = B.sample(u0, u1, wo, wi, p);
                nd = to_world(fr, wi);
            }
            if (guided) p = cont_pdf(nd, wi);
            if (record && guidable(B)) {  // also in the first, BSDF-only pass
                const int64_t rs = (int64_t)path * R.depth + depth;
                for (int k = 0; k < 5; ++k) R.feat[rs * 5 + k] = feat[j * 5 + k];
                R.dir[rs * 3] = nd.x;
                R.dir[rs * 3 + 1] = nd.y;
                R.dir[rs * 3 + 2] = nd.z;
                R.thr[rs * 3] = thr.x;
                R.thr[rs * 3 + 1] = thr.y;
                R.thr[rs * 3 + 2] = thr.z;
                R.res[rs * 3] = res.x;
                R.res[rs * 3 + 1] = res.y;
                R.res[rs * 3 + 2] = res.z;
                R.valid[rs] = 1;
            }
            f3 no = pos + nd * 0.001f;
            if (all_zero(f) || !(p > 0.f)) thr = mk(0, 0, 0);
            else thr = thr * f * fabsf(dot3(nd, nrm)) / p;
            next_pdf = p;
            next_delta = B.is_delta();
            if (!all_zero(thr) && finite3(thr)) {
                cont = true;
                next = cav_ray{no.x, no.y, no.z, 0.f, nd.x, nd.y, nd.z, INFINITY};
            }
        }
    }
    if (valid && !hit && S.env >= 0) {  // rays leaving the scene see the environment
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

// evalMaterial's accumulation; an unoccluded light sample also belongs to the radiance
// recorded "before the continuation" at its vertex
__global__ void k_g_add_direct(int64_t n, Paths P, Queues Q, Records R, int depth, int record) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (Q.shadow_occ[k] != 0) return;
    int path = Q.shadow_path[k];
    const float c0 = Q.shadow_contrib[3 * k], c1 = Q.shadow_contrib[3 * k + 1], c2 = Q.shadow_contrib[3 * k + 2];
    P.result[3 * path] += c0;
    P.result[3 * path + 1] += c1;
    P.result[3 * path + 2] += c2;
    if (record) {
        const int64_t rs = (int64_t)path * R.depth + depth;
        if (R.valid[rs]) {
            R.res[rs * 3] += c0;
            R.res[rs * 3 + 1] += c1;
            R.res[rs * 3 + 2] += c2;
        }
    }
}

// After a chunk: each recorded vertex becomes a training sample (features, direction,
// luminance of (final radiance - radiance before the continuation) / throughput).
__global__ void k_g_collect(int64_t m, Paths P, Records R, TrainBuf T) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m * R.depth) return;
    if (!R.valid[i]) return;
    R.valid[i] = 0;
    const int64_t path = i / R.depth;
    float w = 0.f;
    for (int c = 0; c < 3; ++c) {
        const float t = R.thr[3 * i + c];
        const float d = P.result[3 * path + c] - R.res[3 * i + c];
        if (t > 0.f) w += (c == 0 ? 0.212671f : c == 1 ? 0.715160f : 0.072169f) * fmaxf(d, 0.f) / t;
    }
    if (!(w > 0.f) || !isfinite(w)) return;
    const uint32_t slot = atomicAdd(T.count, 1u) % T.cap;  // a ring: the newest vertices replace the oldest
    for (int k = 0; k < 5; ++k) T.feat[(int64_t)slot * 5 + k] = R.feat[i * 5 + k];
    for (int k = 0; k < 3; ++k) T.dir[(int64_t)slot * 3 + k] = R.dir[i * 3 + k];
    T.w[slot] = w;
}

// Loss weights are heavy-tailed (a few vertices see the light through a small opening):
// scale them to mean 1 over the training set and clip at 20.
__global__ void k_g_weight_sum(const float* w, uint32_t n, float* sum) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float v = i < n ? w[i] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, v);
}
__global__ void k_g_weight_norm(float* w, uint32_t n, const float* sum) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float mean = *sum / (float)n;
    if (mean > 0.f) w[i] = fminf(w[i] / mean, 20.f);
}

}  // namespace

cav_status render_guided(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                         cudaStream_t s, cav_mlp* net, const cav_guide_opts* gopt, cav_guide_stats* gstats) {
    const cavpbrt::Scene& D = sc->desc;
    int W, H;
    film_size(sc, opts, W, H);
    const int spp_total = opts && opts->spp > 0 ? opts->spp : D.spp;
    const int max_depth = opts && opts->max_depth > 0 ? opts->max_depth : D.max_depth;
    const int64_t pixels = (int64_t)W * H;
    int64_t chunk = opts && opts->max_paths_in_flight > 0 ? opts->max_paths_in_flight : (int64_t)1 << 22;
    // passes render 1, 1, 2, 4, ... samples per pixel: the largest pass bounds the paths in flight
    int max_pass = 1;
    for (int done = 0, p = 0, ps = 1; done < spp_total; ++p) {
        max_pass = std::max(max_pass, std::min(ps, spp_total - done));
        done += std::min(ps, spp_total - done);
        if (p >= 1) ps *= 2;
    }
    chunk = std::min(chunk, pixels * max_pass);
    const float alpha = gopt && gopt->alpha > 0.f ? gopt->alpha : 0.5f;
    const uint32_t cap = gopt && gopt->train_samples_per_pass > 0 ? (uint32_t)gopt->train_samples_per_pass : (1u << 18);
    const int steps_per_pass = gopt && gopt->train_steps_per_pass > 0 ? gopt->train_steps_per_pass : 32;
    const int batch = gopt && gopt->train_batch > 0 ? gopt->train_batch : 16384;
    const float lr = gopt && gopt->learning_rate > 0.f ? gopt->learning_rate : 3e-3f;
    const bool train = !(gopt && gopt->freeze);
    size_t need = 0;
    auto acc = [&](size_t bytes) { need += bytes + 256; };
    acc(8 * chunk); acc(8 * chunk); acc(12 * chunk); acc(12 * chunk); acc(4 * chunk); acc(chunk);
    acc(4 * chunk); acc(32 * chunk); acc(4 * chunk); acc(32 * chunk);
    acc(4 * chunk); acc(4 * chunk); acc(8 * chunk);
    acc(32 * chunk); acc(4 * chunk); acc(8 * chunk); acc(4 * chunk); acc(12 * chunk); acc(chunk); acc(64);
    acc(20 * chunk); acc(128 * chunk);                           // features, network outputs
    acc((size_t)chunk * max_depth * (20 + 12 + 12 + 12 + 1));    // records
    acc((size_t)cap * (20 + 12 + 4)); acc(16); acc(16);          // training buffer
    void* base = nullptr;
    CAV_CUDA(ctx, cudaMallocAsync(&base, need, s));
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
    float* feat = carve<float>(p, 5 * chunk);
    float* mout = carve<float>(p, 32 * chunk);
    Records R;
    R.depth = max_depth;
    R.feat = carve<float>(p, (size_t)5 * chunk * max_depth);
    R.dir = carve<float>(p, (size_t)3 * chunk * max_depth);
    R.thr = carve<float>(p, (size_t)3 * chunk * max_depth);
    R.res = carve<float>(p, (size_t)3 * chunk * max_depth);
    R.valid = carve<uint8_t>(p, (size_t)chunk * max_depth);
    TrainBuf T;
    float* wsum = carve<float>(p, 4);
    T.feat = carve<float>(p, (size_t)5 * cap);
    T.dir = carve<float>(p, (size_t)3 * cap);
    T.w = carve<float>(p, cap);
    T.count = carve<uint32_t>(p, 4);
    T.cap = cap;
    CAV_CUDA(ctx, cudaMemsetAsync(R.valid, 0, (size_t)chunk * max_depth, s));
    CAV_CUDA(ctx, cudaMemsetAsync(T.count, 0, 4, s));
    uint32_t have = 0;  // training vertices in the ring (all passes so far)

    const DevScene S = dev_scene_of(sc);
    const Camera cam = camera_of(sc, W, H);
    const float* box = sc->bvh->d_root_box;
    auto& log = sc->log;
    log.reset();
    log.start = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.start, s));
    log.paths = pixels * spp_total;
    cav_guide_stats gs{};
    uint32_t counts[2];
    // passes of 1, 1, 2, 4, ... samples per pixel (the sample index continues across passes)
    int done_spp = 0, pass = 0, pass_spp = 1;
    while (done_spp < spp_total) {
        const int this_spp = std::min(pass_spp, spp_total - done_spp);
        // the network is sampled once it has been trained on a few thousand vertices
        const float a = (pass == 0 || (train && have < 4096)) ? 0.f : alpha;
        const int record = train && done_spp + this_spp < spp_total;
        const int64_t total = pixels * this_spp;
        for (int64_t first = 0; first < total; first += chunk) {
            const int64_t m = std::min(chunk, total - first);
            // samples of this pass: pixel-major over this_spp, with indices offset by done_spp
            k_generate_pass<<<div_up(m, kThreads), kThreads, 0, s>>>(cam, S.halton, spp_total, this_spp, done_spp,
                                                                     first, m, P, Q);
            int64_t n = m;
            int dim0 = 0;
            for (int depth = 0; n > 0 && depth < max_depth; ++depth) {
                cav_status st = trace_closest(ctx, sc->bvh, Q.rays, n, Q.hit_prim, Q.hit_t, Q.hit_uv, CAV_TRACE_EXACT,
                                              s, ctx->d_counters + 6);
                if (st != CAV_OK) return st;
                k_g_features<<<div_up(n, kThreads), kThreads, 0, s>>>(S, box, n, Q, feat);
                if (a > 0.f) {
                    st = mlp_forward(net, feat, n, mout, s);
                    if (st != CAV_OK) return st;
                }
                CAV_CUDA(ctx, cudaMemsetAsync(Q.counters, 0, 8, s));
                k_g_shade<<<div_up(n, kThreads), kThreads, 0, s>>>(S, depth, dim0, n, P, Q, feat, mout, a, R, record);
                CAV_CUDA(ctx, cudaMemcpyAsync(counts, Q.counters, 8, cudaMemcpyDeviceToHost, s));
                CAV_CUDA(ctx, cudaStreamSynchronize(s));
                log.closest_rays += n;
                log.shadow_rays += counts[1];
                log.bounces = std::max(log.bounces, depth + 1);
                if (counts[1] > 0) {
                    st = trace_any(ctx, sc->bvh, Q.shadow_rays, Q.shadow_limit, Q.shadow_excl, counts[1],
                                   Q.shadow_occ, CAV_TRACE_EXACT, s, ctx->d_counters + 7);
                    if (st != CAV_OK) return st;
                    k_g_add_direct<<<div_up(counts[1], kThreads), kThreads, 0, s>>>(counts[1], P, Q, R, depth, record);
                }
                std::swap(Q.active, Q.next_active);
                std::swap(Q.rays, Q.next_rays);
                n = counts[0];
                dim0 += kDims;
            }
            if (record)
                k_g_collect<<<div_up(m * max_depth, kThreads), kThreads, 0, s>>>(m, P, R, T);
            k_film<<<div_up(m, kThreads), kThreads, 0, s>>>(m, P, W, H, D.filter_xwidth, D.filter_ywidth, d_sum,
                                                             d_wsum);
        }
        if (record) {  // train on the ring of vertices before the next pass samples the network
            uint32_t total_seen = 0;
            CAV_CUDA(ctx, cudaMemcpyAsync(&total_seen, T.count, 4, cudaMemcpyDeviceToHost, s));
            CAV_CUDA(ctx, cudaStreamSynchronize(s));
            gs.train_samples = total_seen;
            have = std::min(total_seen, cap);
            if (have >= 256) {
                CAV_CUDA(ctx, cudaMemsetAsync(wsum, 0, 4, s));
                k_g_weight_sum<<<div_up(have, kThreads), kThreads, 0, s>>>(T.w, have, wsum);
                k_g_weight_norm<<<div_up(have, kThreads), kThreads, 0, s>>>(T.w, have, wsum);
                for (int k = 0; k < steps_per_pass; ++k) {
                    const int64_t bsz = std::min<int64_t>(batch, have);
                    const int64_t off = ((int64_t)k * bsz) % (have - bsz + 1);
                    cav_status st = cav_mlp_train_step(net, T.feat + off * 5, T.dir + off * 3, T.w + off, bsz, lr, s);
                    if (st != CAV_OK) return st;
                    gs.train_steps += 1;
                }
                CAV_CUDA(ctx, cudaStreamSynchronize(s));
                cav_mlp_last_loss(net, &gs.last_loss);
            }
        }
        gs.passes += 1;
        done_spp += this_spp;
        pass += 1;
        if (pass >= 2) pass_spp *= 2;
    }
    CAV_CUDA(ctx, cudaGetLastError());
    log.end = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.end, s));
    if (gstats) *gstats = gs;
    return CAV_OK;
}

}  // namespace cav

extern "C" cav_status cav_render_guided(cav_ctx* ctx, cav_scene* scene, const cav_render_opts* opts, cav_mlp* mlp,
                                        const cav_guide_opts* gopts, float* film_sum, float* film_weight, void* stream,
                                        cav_guide_stats* stats) {
    if (!ctx || !scene || !film_sum || !film_weight) return CAV_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return cav::cuda_error(ctx, cudaGetLastError(), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    int W, H;
    cav::film_size(scene, opts, W, H);
    const int64_t pixels = (int64_t)W * H;
    CAV_CUDA(ctx, cudaMemsetAsync(film_sum, 0, sizeof(float) * 3 * pixels, s));
    CAV_CUDA(ctx, cudaMemsetAsync(film_weight, 0, sizeof(float) * pixels, s));
    cav_mlp* net = mlp;
    if (!net) {
        cav_status st = cav_mlp_create(ctx, gopts && gopts->seed ? gopts->seed : 1, &net);
        if (st != CAV_OK) return st;
    }
    cav_status st = cav::render_guided(ctx, scene, opts, film_sum, film_weight, s, net, gopts, stats);
    if (!mlp) {
        cudaStreamSynchronize(s);
        cav_mlp_free(net);
    }
    return st;
}
