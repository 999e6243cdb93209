// Reinforcement-learning path integrator for sm_100a: the reference's rlpath
// (Integrators/ReinforcementLearningPathTracing.cu), a path tracer whose continuation
// directions are drawn from a learned radiance table instead of the BSDF alone.
//
// The table has 32^3 spatial entries over the scene box (findQEntry, :164-174), each with
// 8 x 16 direction cells over the whole sphere (QEntry, :10-148; cell index = theta * 16 +
// phi, dirToCellIndex :113-128).  Per bounce every hit:
//   * samples a light from a per-entry learned light distribution (computeLighting
//     :387-460) and traces its shadow ray;
//   * evaluates Q * f * |cos| in all 128 cells (computeQDistributions :516-606), proposes
//     that sum (+ emission seen) as the new Q of the cell the path came through (SARSA),
//     proposes the directly sampled light to its own cell, and samples the next cell;
//   * adds the light sample MIS-weighted against the Q pdf (accumulateLightingContribs
//     :608-647).
// After every bounce the proposals are folded in with a count-based learning rate
// (finishUpdateQ, averageQ :737-767) and the light distributions retrained
// (finishLightingTraining :462-514).  Delta and near-delta BSDFs, and hits with an
// all-zero table product, continue by BSDF sampling (genNextRay :304-375).
//
// The table is SoA in HBM (Q, newQ, proposal counts, totals: 4 x 4 B x 4.2M cells = 64 MiB),
// persists across the chunks of a render, and is updated with float/int atomics as in
// the reference, so results are not bit-reproducible run to run (the reference's are not
// either).  Halton dimensions follow the reference's per-queue maximum (syncDimension,
// :281-315): the dimension base of each stage is the maximum any task of the queue reached.
// Unlike the path integrator, paths whose throughput is zero are kept: they still propose
// table values and light statistics.
#include <cstdio>
#include <cstring>

#include "render_common.cuh"

namespace cav {
namespace {

constexpr int kQRes = 32;                      // Q_TABLE_SIZE
constexpr int kEntries = kQRes * kQRes * kQRes;
constexpr int kNumX = 16, kNumY = 8;           // QEntry::NUM_X / NUM_Y
constexpr int kCells = kNumX * kNumY;
// QEntry's cell solid angle: constexpr float (4.f * M_PI / (float)NUM_XY), a double
// expression rounded once to float
constexpr float kCellSolidAngle = (float)(4.f * 3.14159265358979323846 / (float)kCells);

struct QTable {
    float* Q;         // kEntries * kCells
    float* newQ;
    int32_t* prop;    // proposalCount
    int32_t* total;   // totalProposalCount
};

struct LightTable {  // per entry x light
    float* cdf;
    float* res;
    int32_t* cnt;
    float* new_res;
    int32_t* new_cnt;
    int n_lights;
};

// per ray slot of the current bounce (indexed like the extend queue)
struct RLTask {
    float* light_dir;    // 3
    float* light_pdf;
    float* incident;     // 3
    float* sel_prob;
    int32_t* light_idx;
    int32_t* entry;
    float* emis_lum;
    uint8_t* occluded;
    uint8_t* shadowed;   // a shadow ray was traced for this slot
    float* next_dir;     // 3
    float* next_pdf;
    int32_t* next_cell;
    uint8_t* next_valid;
};

struct RLPath {  // per path
    int32_t* prev_entry;
    int32_t* prev_cell;
    int32_t* dim;
};

__device__ inline float luminance(f3 c) { return dot3(c, mk(0.212671f, 0.715160f, 0.072169f)); }

// findQEntry (:164-174)
__device__ inline int find_entry(const float* box, f3 p) {
    f3 lo = mk(box[0], box[1], box[2]), hi = mk(box[3], box[4], box[5]);
    f3 size = hi - lo;
    f3 es = mk(size.x / (float)kQRes, size.y / (float)kQRes, size.z / (float)kQRes);
    p = p - lo;
    int ex = min(max((int)(p.x / es.x), 0), kQRes - 1);
    int ey = min(max((int)(p.y / es.y), 0), kQRes - 1);
    int ez = min(max((int)(p.z / es.z), 0), kQRes - 1);
    return ex * kQRes * kQRes + ey * kQRes + ez;
}

// QEntry::dirToCellIndex (:113-128)
__device__ inline int dir_to_cell(f3 dir) {
    float u = dir.z;
    float y = (u + 1.f) / 2.f;
    int theta = min(max((int)(y * kNumY), 0), kNumY - 1);
    dir.x /= sqrtf(1.f - u * u);
    dir.y /= sqrtf(1.f - u * u);
    float v = acosf(dir.x);
    if (dir.y < 0) v = (float)((2.f * 3.14159265358979323846) - v);
    v = (float)(v / (2.f * 3.14159265358979323846));
    int phi = min(max((int)(v * kNumX), 0), kNumX - 1);
    return theta * kNumX + phi;
}

// QEntry::sampleDirectionInCell (:131-147)
__device__ inline f3 dir_in_cell(float r0, float r1, int cell) {
    int ti = cell / kNumX, pi = cell % kNumX;
    float u = ((float)ti + r0) * (1.f / (float)kNumY);
    u = u * 2 - 1.f;
    float v = ((float)pi + r1) * (1.f / (float)kNumX);
    float xy = sqrtf(1.0f - u * u);
    float phi = (float)(2 * 3.14159265358979323846 * v);
    return mk(xy * cosf(phi), xy * sinf(phi), u);
}

// Distribution1D::getCorrespondingIndex / sample / pdf (Utils/RandomUtils.h:120-184)
__device__ inline int cdf_index(const float* cdf, int n, float f) {
    int l = 0, r = n - 1;
    while (l < r) {
        int m = (l + r) / 2;
        if (cdf[m] >= f) {
            if (m == 0) return 0;
            if (cdf[m - 1] < f) return m;
            r = m - 1;
        } else {
            l = m + 1;
        }
    }
    return l;
}
__device__ inline int cdf_sample(const float* cdf, int n, float u, float& prob) {
    int i = cdf_index(cdf, n, u);
    prob = cdf[i];
    if (i > 0) prob -= cdf[i - 1];
    return i;
}
__device__ inline float cdf_pdf(const float* cdf, int i) { return i == 0 ? cdf[0] : cdf[i] - cdf[i - 1]; }

// isAlmostDelta (BSDFs/MicrofacetDistribution.h:157-159) is overridden by MicrofacetBSDF
// (metal, rough glass) and FresnelBlend (substrate): alpha_x < 0.05 or alpha_y < 0.05.
__device__ inline bool almost_delta(const Bsdf& B) {
    const bool microfacet = B.type == cavpbrt::kMetal || B.type == cavpbrt::kSubstrate ||
                            (B.type == cavpbrt::kGlass && B.rough());
    return microfacet && (B.ggx.ax < 0.05f || B.ggx.ay < 0.05f);
}

// Hit geometry of extend slot j, recomputed where needed (Triangle::fillIntersectionInformation).
struct Hit {
    f3 ro, rd, pos, nrm;
    int mesh;
    int prim;
    float u, v;
};
__device__ inline Hit hit_of(const DevScene& S, const Queues& Q, int64_t j, int prim) {
    const cav_ray r = Q.rays[j];
    Hit h;
    h.ro = mk(r.ox, r.oy, r.oz);
    h.rd = mk(r.dx, r.dy, r.dz);
    h.pos = h.ro + Q.hit_t[j] * h.rd;
    h.mesh = S.tri_mesh[prim];
    h.prim = prim;
    h.u = Q.hit_uv[2 * j];
    h.v = Q.hit_uv[2 * j + 1];
    h.nrm = tri_normal(S, S.meshes[h.mesh], prim, h.u, h.v);
    return h;
}

__global__ void k_rl_init(int64_t n, RLPath R) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    R.prev_entry[i] = -1;
    R.prev_cell[i] = -1;
    R.dim[i] = 0;
}

// syncDimension before computeLighting: the maximum dimension over the hit tasks.
__global__ void k_rl_dim_max(int64_t n, Queues Q, RLPath R, int32_t* dim_max) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int d = -1;
    if (j < n && Q.hit_prim[j] >= 0) d = R.dim[Q.active[j]];
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0 && d >= 0) atomicMax(dim_max, d);
}

// computeLighting (:387-460) up to the visibility test: emission with MIS, light choice
// from the entry's learned distribution, rand4 (unused), the light-surface sample.  The
// shadow ray is queued when it can change the result (non-zero incident radiance with a
// finite pdf); otherwise the reference's occluded branch applies regardless of visibility.
__global__ void k_rl_light(DevScene S, const float* box, LightTable LT, int depth, const int32_t* dim_in, int64_t n,
                           Paths P, Queues Q, RLTask T, RLPath R) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int prim = j < n ? Q.hit_prim[j] : -1;
    bool emit = false;
    cav_ray shadow{};
    float limit = 0.f;
    int2 excl = make_int2(-1, -1);
    if (prim >= 0) {
        const int path = Q.active[j];
        const Hit h = hit_of(S, Q, j, prim);
        const uint64_t index = P.sample_index[path];
        const f3 thr = ld3(P.throughput + 3 * path);
        f3 res = ld3(P.result + 3 * path);
        const RMesh& M = S.meshes[h.mesh];
        float emis = 0.f;
        if (M.light >= 0) {
            const RLight& L = S.lights[M.light];
            f3 Le = dot3(h.rd, h.nrm) >= 0 ? mk(0, 0, 0) : ld3(L.L);
            if (P.delta[path]) {
                res = res + Le * thr;
            } else if (depth > 0) {
                float light_pdf = light_surface_pdf(S.meshes[L.mesh], h.ro, h.pos, h.nrm);
                float w = mis_power(P.mat_pdf[path], light_pdf);
                if (isfinite(w)) {
                    emis = luminance(Le);
                    res = res + Le * thr * w;
                }
            }
        }
        P.result[3 * path] = res.x;
        P.result[3 * path + 1] = res.y;
        P.result[3 * path + 2] = res.z;
        const int entry = find_entry(box, h.pos);
        int dim = *dim_in;
        float sel = 0.f;
        const int li = cdf_sample(LT.cdf + (int64_t)entry * LT.n_lights, LT.n_lights, halton(S.halton, index, dim), sel);
        dim += 4;  // rand4, drawn and unused
        const LightSample ls = sample_light(S, S.lights[li], h.pos, index, dim);
        // computeQDistributions draws from this path's own state, which the reference does
        // not synchronise after computeLighting: 2 (environment, sphere cone) or 3 (triangle)
        // light-sample dimensions on from here
        R.dim[path] = dim;
        const float light_pdf = ls.pdf;
        const f3 dir = ls.dir;
        const f3 incident = ls.incident;
        T.light_dir[3 * j] = dir.x;
        T.light_dir[3 * j + 1] = dir.y;
        T.light_dir[3 * j + 2] = dir.z;
        T.light_pdf[j] = light_pdf;
        T.incident[3 * j] = incident.x;
        T.incident[3 * j + 1] = incident.y;
        T.incident[3 * j + 2] = incident.z;
        T.sel_prob[j] = sel;
        T.light_idx[j] = li;
        T.entry[j] = entry;
        T.emis_lum[j] = emis;
        T.occluded[j] = 0;
        emit = !all_zero(incident) && isfinite(light_pdf);
        T.shadowed[j] = emit ? 1 : 0;
        if (emit) {
            shadow = cav_ray{h.pos.x, h.pos.y, h.pos.z, 0.f, dir.x, dir.y, dir.z, INFINITY};
            limit = ls.dist;
            excl = make_int2(h.mesh, ls.target);
        }
    } else if (j < n && S.env >= 0) {  // intersectScene :292-296: the environment, no MIS weight
        const int path = Q.active[j];
        const cav_ray r = Q.rays[j];
        const f3 e = env_eval(S, S.lights[S.env], mk(r.dx, r.dy, r.dz)) * ld3(P.throughput + 3 * path);
        P.result[3 * path] += e.x;
        P.result[3 * path + 1] += e.y;
        P.result[3 * path + 2] += e.z;
    }
    uint32_t k = warp_append(Q.counters + 1, emit);
    if (emit) {
        Q.shadow_rays[k] = shadow;
        Q.shadow_limit[k] = limit;
        reinterpret_cast<int2*>(Q.shadow_excl)[k] = excl;
        Q.shadow_path[k] = (int32_t)j;  // the extend slot, not the path
    }
}

__global__ void k_rl_occlusion(int64_t m, Queues Q, RLTask T) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    T.occluded[Q.shadow_path[k]] = Q.shadow_occ[k] != 0;
}

// The end of computeLighting (light statistics), computeQDistributions and
// accumulateLightingContribs for one hit.  dim_out receives the maximum dimension reached
// (syncDimension before genNextRay).
// 6 blocks of 128 per SM (80 registers, a few bytes spilled) rather than 4 at 117: more
// resident warps for a kernel that waits on the Q-table and light-table loads (with the
// k_rl_next bound below: 640x360 64-spp rlpath render of the aperture scene 179 -> 172 ms)
__global__ void __launch_bounds__(128, 6) k_rl_q(DevScene S, QTable QT, LightTable LT, const int32_t* dim_in, int64_t n,
                                              Paths P, Queues Q, RLTask T, RLPath R, int32_t* dim_out) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int prim = j < n ? Q.hit_prim[j] : -1;
    if (prim < 0) return;
    const int path = Q.active[j];
    const Hit h = hit_of(S, Q, j, prim);
    const uint64_t index = P.sample_index[path];
    const RMesh& M = S.meshes[h.mesh];
    const Bsdf B = material_bsdf(S, S.mats[M.material], h.prim, h.u, h.v);
    const Frame fr = make_frame(h.nrm);
    const f3 wo = to_local(fr, h.rd * -1.f);
    // ---- light result: occluded (or non-finite pdf) samples carry zero radiance, pdf 1
    f3 ldir = ld3(T.light_dir + 3 * j);
    f3 incident = ld3(T.incident + 3 * j);
    float lpdf = T.light_pdf[j];
    if ((T.shadowed[j] && T.occluded[j]) || !isfinite(lpdf)) {
        incident = mk(0, 0, 0);
        lpdf = 1;
    }
    const f3 wl = to_local(fr, ldir);
    f3 contrib = incident * B.eval(wl, wo) * fabsf(dot3(ldir, h.nrm));  // Material::eval
    contrib = contrib * (1.f / (lpdf * T.sel_prob[j]));
    const int entry = T.entry[j];
    const int64_t ls = (int64_t)entry * LT.n_lights + T.light_idx[j];
    const float sampled = luminance(incident);
    atomicAdd(LT.new_res + ls, sampled);
    atomicAdd(LT.new_cnt + ls, 1);
    // ---- Q distribution over the 128 cells of this entry
    int dim = R.dim[path];  // after this path's light sample (k_rl_light)
    const float r0 = halton(S.halton, index, dim);
    const float r1 = halton(S.halton, index, dim);
    const float* q = QT.Q + (int64_t)entry * kCells;
    float cdf[kCells];
    float sum = 0.f;
#pragma unroll 4
    for (int c = 0; c < kCells; ++c) {
        f3 d = dir_in_cell(r0, r1, c);
        float scattering = luminance(B.eval(to_local(fr, d), wo));
        sum += fabsf(dot3(d, h.nrm)) * scattering * q[c];
        cdf[c] = sum;
    }
    for (int c = 0; c < kCells; ++c) cdf[c] /= sum;
    sum *= kCellSolidAngle;
    // SARSA proposal for the cell the path arrived through
    const int pe = R.prev_entry[path];
    if (pe != -1) {
        const int64_t pc = (int64_t)pe * kCells + R.prev_cell[path];
        atomicAdd(QT.newQ + pc, sum + T.emis_lum[j]);
        atomicAdd(QT.prop + pc, 1);
    }
    const int lcell = dir_to_cell(ldir);
    float pdf_q = 0.f;
    if (sum != 0) pdf_q = cdf_pdf(cdf, lcell) / kCellSolidAngle;
    // the directly sampled light proposes its own cell
    if (sampled > 0) {
        float esa = 1.f / lpdf;
        float ratio = fminf(1.f, 0.5f * esa / kCellSolidAngle);
        float proposal = sampled * ratio;
        const int64_t tc = (int64_t)entry * kCells + lcell;
        if (proposal > q[lcell]) {
            atomicAdd(QT.newQ + tc, proposal);
            atomicAdd(QT.prop + tc, 1);
        }
    }
    // next direction from the table
    if (sum != 0) {
        float prob = 0.f;
        const int cell = cdf_sample(cdf, kCells, halton(S.halton, index, dim), prob);
        T.next_pdf[j] = (float)(kCells * prob / (4 * 3.14159265358979323846));
        f3 nd = dir_in_cell(r0, r1, cell);
        T.next_dir[3 * j] = nd.x;
        T.next_dir[3 * j + 1] = nd.y;
        T.next_dir[3 * j + 2] = nd.z;
        T.next_cell[j] = cell;
        T.next_valid[j] = 1;
    } else {
        T.next_valid[j] = 0;
    }
    // accumulateLightingContribs
    const float mpdf = B.pdf(wl, wo);
    float spdf = sum != 0 ? pdf_q : 0.f;
    if (sum == 0 || spdf == 0 || B.is_delta() || almost_delta(B)) spdf = mpdf;
    const float w = mis_power(lpdf, spdf);
    const f3 thr = ld3(P.throughput + 3 * path);
    const f3 add = contrib * thr * w;
    P.result[3 * path] += add.x;
    P.result[3 * path + 1] += add.y;
    P.result[3 * path + 2] += add.z;
    atomicMax(dim_out, dim);
}

// QEntry::finishUpdateQ (:98-108): count-based learning rate alpha = n / (N + n)
__global__ void k_rl_finish_q(QTable QT) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)kEntries * kCells) return;
    const int p = QT.prop[i];
    if (p == 0) return;
    const float a = ((float)p) / (float)(QT.total[i] + p);
    if (a == 0) return;
    QT.Q[i] = QT.Q[i] * (1.f - a) + a * QT.newQ[i] / (float)p;
    QT.total[i] += p;
}

// QEntry::averageQ (:53-73): cells never proposed take the mean of the proposed ones
__global__ void k_rl_average_q(QTable QT) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kEntries) return;
    float* q = QT.Q + (int64_t)e * kCells;
    const int32_t* tot = QT.total + (int64_t)e * kCells;
    float sum = 0;
    int count = 0;
    for (int c = 0; c < kCells; ++c)
        if (tot[c] > 0) {
            sum += q[c];
            count += 1;
        }
    if (count == 0) return;
    const float avg = sum / (float)count;
    for (int c = 0; c < kCells; ++c)
        if (tot[c] == 0) q[c] = avg;
}

// finishLightingTraining (:462-514): running mean of the luminance each light delivered
// from this entry, then a new light CDF (unseen lights get the mean, seen-but-dark ones
// the mean over their count)
__global__ void k_rl_finish_lights(LightTable LT) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kEntries) return;
    const int nl = LT.n_lights;
    const int64_t b = (int64_t)e * nl;
    float sum = 0, valid = 0;
    for (int i = 0; i < nl; ++i) {
        int& cnt = LT.cnt[b + i];
        int& ncnt = LT.new_cnt[b + i];
        float& res = LT.res[b + i];
        float& nres = LT.new_res[b + i];
        if (ncnt > 0) {
            float tc = cnt + ncnt;
            res = ((float)cnt / tc) * res + ((float)ncnt / tc) * (nres / (float)ncnt);
            cnt += ncnt;
            sum += res;
            valid += 1;
        }
        ncnt = 0;
        nres = 0;
    }
    if (sum > 0) {
        const float avg = sum / (float)valid;
        float dens = 0;
        for (int i = 0; i < nl; ++i) {
            const int cnt = LT.cnt[b + i];
            const float res = LT.res[b + i];
            if (res > 0) dens += res;
            else if (cnt > 0) dens += avg / (float)cnt;
            else dens += avg;
            LT.cdf[b + i] = dens;
        }
        for (int i = 0; i < nl; ++i) LT.cdf[b + i] /= dens;
    }
}

__global__ void k_rl_init_tables(QTable QT, LightTable LT) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (int64_t)kEntries * kCells) {
        QT.Q[i] = 1.f;  // QEntry::defaultQ
        QT.total[i] = 0;
    }
    if (i < (int64_t)kEntries * LT.n_lights) {  // initialiseLightSamplingDist: uniform CDF
        const int l = (int)(i % LT.n_lights);
        LT.cdf[i] = ((float)l + 1.f) / (float)LT.n_lights;
    }
}

// genNextRay (:304-375): Russian roulette, then the table's direction (with its pdf) or,
// for delta BSDFs and hits without a table product, a BSDF sample.
// 4 blocks per SM (64 registers, a few bytes spilled) rather than 3 at 76
__global__ void __launch_bounds__(kThreads, 4) k_rl_next(DevScene S, int depth, const int32_t* dim_in, int64_t n, Paths P, Queues Q, RLTask T,
                          RLPath R) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int prim = j < n ? Q.hit_prim[j] : -1;
    bool cont = false;
    int path = 0;
    cav_ray next{};
    f3 thr = mk(0, 0, 0);
    float next_pdf = 0.f;
    bool next_delta = false;
    int entry = -1, cell = -1, dim = 0;
    if (prim >= 0) {
        path = Q.active[j];
        const Hit h = hit_of(S, Q, j, prim);
        const uint64_t index = P.sample_index[path];
        thr = ld3(P.throughput + 3 * path);
        dim = *dim_in;
        bool alive = true;
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
            const Bsdf B = material_bsdf(S, S.mats[S.meshes[h.mesh].material], h.prim, h.u, h.v);
            const Frame fr = make_frame(h.nrm);
            const f3 wo = to_local(fr, h.rd * -1.f);
            entry = T.entry[j];
            f3 f, nd;
            float p = 0.f;
            if (B.is_delta() || almost_delta(B) || !T.next_valid[j]) {
                float u0 = halton(S.halton, index, dim);
                float u1 = halton(S.halton, index, dim);
                f3 wi;
                f = B.sample(u0, u1, wo, wi, p);
                nd = to_world(fr, wi);
                cell = dir_to_cell(nd);
            } else {
                cell = T.next_cell[j];
                p = T.next_pdf[j];
                nd = ld3(T.next_dir + 3 * j);
                f = B.eval(to_local(fr, nd), wo);
            }
            if (all_zero(f)) thr = mk(0, 0, 0);
            else thr = thr * f * fabsf(dot3(nd, h.nrm)) / p;
            const f3 no = h.pos + nd * 0.001f;
            next = cav_ray{no.x, no.y, no.z, 0.f, nd.x, nd.y, nd.z, INFINITY};
            next_pdf = p;
            next_delta = B.is_delta();
            cont = true;
        }
    }
    uint32_t k = warp_append(Q.counters + 0, cont);
    if (cont) {
        Q.next_active[k] = path;
        Q.next_rays[k] = next;
        P.throughput[3 * path] = thr.x;
        P.throughput[3 * path + 1] = thr.y;
        P.throughput[3 * path + 2] = thr.z;
        P.mat_pdf[path] = next_pdf;
        P.delta[path] = next_delta ? 1 : 0;
        R.prev_entry[path] = entry;
        R.prev_cell[path] = cell;
        R.dim[path] = dim;
    }
}

}  // namespace

cav_status render_rlpath(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                         cudaStream_t s) {
    const cavpbrt::Scene& D = sc->desc;
    const int spp = opts && opts->spp > 0 ? opts->spp : D.spp;
    const int max_depth = opts && opts->max_depth > 0 ? opts->max_depth : D.max_depth;
    int W, H;
    film_size(sc, opts, W, H);
    const int64_t pixels = (int64_t)W * H;
    const int64_t total = pixels * spp;
    int64_t chunk = opts && opts->max_paths_in_flight > 0 ? opts->max_paths_in_flight : (int64_t)1 << 22;
    chunk = std::min(chunk, total);
    const int nl = (int)D.lights.size();
    const int64_t cells = (int64_t)kEntries * kCells;
    const int64_t lcells = (int64_t)kEntries * nl;
    size_t need = 0;
    auto acc = [&](size_t bytes) { need += bytes + 256; };
    // path state + queues (as the path integrator) + rlpath per-path and per-slot arrays
    acc(8 * chunk); acc(8 * chunk); acc(12 * chunk); acc(12 * chunk); acc(4 * chunk); acc(chunk);
    acc(4 * chunk); acc(32 * chunk); acc(4 * chunk); acc(32 * chunk);
    acc(4 * chunk); acc(4 * chunk); acc(8 * chunk);
    acc(32 * chunk); acc(4 * chunk); acc(8 * chunk); acc(4 * chunk); acc(12 * chunk); acc(chunk); acc(64);
    acc(12 * chunk); acc(4 * chunk); acc(12 * chunk); acc(4 * chunk); acc(4 * chunk); acc(4 * chunk); acc(4 * chunk);
    acc(chunk); acc(chunk); acc(12 * chunk); acc(4 * chunk); acc(4 * chunk); acc(chunk);
    acc(12 * chunk);
    acc(16 * cells);
    acc(20 * lcells);
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
    RLTask T;
    T.light_dir = carve<float>(p, 3 * chunk);
    T.light_pdf = carve<float>(p, chunk);
    T.incident = carve<float>(p, 3 * chunk);
    T.sel_prob = carve<float>(p, chunk);
    T.light_idx = carve<int32_t>(p, chunk);
    T.entry = carve<int32_t>(p, chunk);
    T.emis_lum = carve<float>(p, chunk);
    T.occluded = carve<uint8_t>(p, chunk);
    T.shadowed = carve<uint8_t>(p, chunk);
    T.next_dir = carve<float>(p, 3 * chunk);
    T.next_pdf = carve<float>(p, chunk);
    T.next_cell = carve<int32_t>(p, chunk);
    T.next_valid = carve<uint8_t>(p, chunk);
    RLPath R;
    R.prev_entry = carve<int32_t>(p, chunk);
    R.prev_cell = carve<int32_t>(p, chunk);
    R.dim = carve<int32_t>(p, chunk);
    QTable QT;
    QT.Q = carve<float>(p, cells);
    QT.newQ = carve<float>(p, cells);
    QT.prop = carve<int32_t>(p, cells);
    QT.total = carve<int32_t>(p, cells);
    LightTable LT;
    LT.n_lights = nl;
    LT.cdf = carve<float>(p, lcells);
    LT.res = carve<float>(p, lcells);
    LT.cnt = carve<int32_t>(p, lcells);
    LT.new_res = carve<float>(p, lcells);
    LT.new_cnt = carve<int32_t>(p, lcells);
    // zero-filled light statistics (GpuArray zero-fills), then the table defaults
    CAV_CUDA(ctx, cudaMemsetAsync(LT.res, 0, sizeof(float) * lcells, s));
    CAV_CUDA(ctx, cudaMemsetAsync(LT.cnt, 0, sizeof(int32_t) * lcells, s));
    CAV_CUDA(ctx, cudaMemsetAsync(LT.new_res, 0, sizeof(float) * lcells, s));
    CAV_CUDA(ctx, cudaMemsetAsync(LT.new_cnt, 0, sizeof(int32_t) * lcells, s));
    k_rl_init_tables<<<div_up(std::max(cells, lcells), kThreads), kThreads, 0, s>>>(QT, LT);
    int32_t* dims = reinterpret_cast<int32_t*>(Q.counters + 4);  // [0] lighting base, [1] next-ray base

    DevScene S = dev_scene_of(sc);
    Camera cam = camera_of(sc, W, H);
    const float* box = sc->bvh->d_root_box;
    uint32_t counts[2];
    auto& log = sc->log;
    log.reset();
    log.start = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.start, s));
    log.paths = total;
    for (int64_t first = 0; first < total; first += chunk) {
        const int64_t m = std::min(chunk, total - first);
        k_generate<<<div_up(m, kThreads), kThreads, 0, s>>>(cam, S.halton, spp, first, m, P, Q);
        k_rl_init<<<div_up(m, kThreads), kThreads, 0, s>>>(m, R);
        int64_t n = m;
        for (int depth = 0; n > 0 && depth < max_depth; ++depth) {
            cudaEvent_t e0 = log.next(), e1 = log.next(), e2 = log.next();
            CAV_CUDA(ctx, cudaEventRecord(e0, s));
            cav_status st = trace_closest(ctx, sc->bvh, Q.rays, n, Q.hit_prim, Q.hit_t, Q.hit_uv, CAV_TRACE_EXACT, s,
                                          ctx->d_counters + 6);
            if (st != CAV_OK) return st;
            CAV_CUDA(ctx, cudaEventRecord(e1, s));
            CAV_CUDA(ctx, cudaMemsetAsync(Q.counters, 0, 32, s));
            CAV_CUDA(ctx, cudaMemsetAsync(QT.newQ, 0, sizeof(float) * cells, s));  // prepareForUpdateQ
            CAV_CUDA(ctx, cudaMemsetAsync(QT.prop, 0, sizeof(int32_t) * cells, s));
            k_rl_dim_max<<<div_up(n, kThreads), kThreads, 0, s>>>(n, Q, R, dims);
            k_rl_light<<<div_up(n, kThreads), kThreads, 0, s>>>(S, box, LT, depth, dims, n, P, Q, T, R);
            CAV_CUDA(ctx, cudaMemcpyAsync(counts, Q.counters, 8, cudaMemcpyDeviceToHost, s));
            CAV_CUDA(ctx, cudaStreamSynchronize(s));
            log.closest.emplace_back(e0, e1);
            log.closest_rays += n;
            log.shadow_rays += counts[1];
            log.bounces = std::max(log.bounces, depth + 1);
            if (counts[1] > 0) {
                cudaEvent_t e3 = log.next(), e4 = log.next();
                CAV_CUDA(ctx, cudaEventRecord(e3, s));
                st = trace_any(ctx, sc->bvh, Q.shadow_rays, Q.shadow_limit, Q.shadow_excl, counts[1], Q.shadow_occ,
                               CAV_TRACE_EXACT, s, ctx->d_counters + 7);
                if (st != CAV_OK) return st;
                CAV_CUDA(ctx, cudaEventRecord(e4, s));
                log.any.emplace_back(e3, e4);
                k_rl_occlusion<<<div_up(counts[1], kThreads), kThreads, 0, s>>>(counts[1], Q, T);
            }
            CAV_CUDA(ctx, cudaEventRecord(e2, s));
            k_rl_q<<<div_up(n, 128), 128, 0, s>>>(S, QT, LT, dims, n, P, Q, T, R, dims + 1);
            k_rl_finish_q<<<div_up(cells, kThreads), kThreads, 0, s>>>(QT);
            k_rl_average_q<<<div_up(kEntries, kThreads), kThreads, 0, s>>>(QT);
            k_rl_finish_lights<<<div_up(kEntries, kThreads), kThreads, 0, s>>>(LT);
            k_rl_next<<<div_up(n, kThreads), kThreads, 0, s>>>(S, depth, dims + 1, n, P, Q, T, R);
            cudaEvent_t e5 = log.next();
            CAV_CUDA(ctx, cudaEventRecord(e5, s));
            log.shade.emplace_back(e2, e5);
            CAV_CUDA(ctx, cudaMemcpyAsync(counts, Q.counters, 4, cudaMemcpyDeviceToHost, s));
            CAV_CUDA(ctx, cudaStreamSynchronize(s));
            std::swap(Q.active, Q.next_active);
            std::swap(Q.rays, Q.next_rays);
            n = counts[0];
        }
        k_film<<<div_up(m, kThreads), kThreads, 0, s>>>(m, P, W, H, D.filter_xwidth, D.filter_ywidth,
                                                         d_sum, d_wsum);
    }
    CAV_CUDA(ctx, cudaGetLastError());
    log.end = log.next();
    CAV_CUDA(ctx, cudaEventRecord(log.end, s));
    return CAV_OK;
}

}  // namespace cav
