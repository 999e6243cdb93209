// Shared device code of the wavefront integrators (render.cu: path, rlpath.cu: rlpath):
// the Halton sampler, local frames, BSDFs, scene records, path state and queues, camera
// sample generation and the film splat; and the host scene object.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cav_internal.cuh"
#include "cav_render.h"
#include "pbrt.h"

namespace cav {
namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr double kPiD = 3.14159265358979323846;
// cosineSampleHemispherePdf: |z / M_PI| in double (Utils/RandomUtils.h:53-56)
__device__ inline float cosine_pdf(float z) { return (float)fabs((double)z / kPiD); }
constexpr int kThreads = 256;
constexpr int kPrimes = 1024;

// ------------------------------------------------------------------- vector helpers
__device__ inline f3 operator*(float s, f3 a) { return a * s; }
__device__ inline f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ inline f3 neg(f3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ inline float length3(f3 a) { return sqrtf(dot3(a, a)); }
__device__ inline f3 normalize3(f3 a) {
    float inv = rsqrtf(dot3(a, a));
    return a * inv;
}
__device__ inline bool all_zero(f3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
__device__ inline bool finite3(f3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ inline f3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

// ------------------------------------------------------------------------ Halton
struct Halton {
    const uint32_t* primes;
    const uint32_t* perm_start;
    const uint16_t* perms;
};

// runHalton + HaltonSampler::rand1 (Samplers/HaltonSampler.h:13-23, :59-66)
__device__ inline float halton(const Halton& h, uint64_t index, int& dim) {
    const int d = dim < kPrimes ? dim : kPrimes - 1;
    dim += 1;
    const uint32_t base = h.primes[d];
    const uint16_t* perm = h.perms + h.perm_start[d];
    float r = 0, f = 1;
    uint64_t i = index;
    while (i > 0) {
        f = f / base;
        r = r + f * (perm[i % base]);
        i = i / base;
    }
    return r;
}
__device__ inline int halton_int(const Halton& h, uint64_t index, int& dim, int N) {
    float f = halton(h, index, dim);
    int r = f * N;
    if (r >= N) r = N - 1;
    return r;
}

// ------------------------------------------------------------------- local frame
struct Frame {
    f3 t0, t1, n;
};
// buildCoordinateSystem (Utils/MathsCommons.h:194-202)
__device__ inline Frame make_frame(f3 n) {
    f3 t0 = fabsf(n.x) < 0.5f ? cross3(mk(1, 0, 0), n) : cross3(mk(0, 1, 0), n);
    t0 = normalize3(t0);
    f3 t1 = normalize3(cross3(n, t0));
    return Frame{t0, t1, n};
}
__device__ inline f3 to_local(const Frame& fr, f3 v) { return mk(dot3(fr.t0, v), dot3(fr.t1, v), dot3(fr.n, v)); }
__device__ inline f3 to_world(const Frame& fr, f3 v) { return fr.t0 * v.x + fr.t1 * v.y + fr.n * v.z; }

__device__ inline bool same_hemisphere(f3 a, f3 b) { return a.z * b.z > 0; }
__device__ inline float pow5(float f) { return (f * f) * (f * f) * f; }
__device__ inline float clampf(float x, float lo, float hi) { return fmaxf(lo, fminf(x, hi)); }
__device__ inline float cos2_theta(f3 w) { return w.z * w.z; }
__device__ inline float sin2_theta(f3 w) { return fmaxf(0.f, 1.f - cos2_theta(w)); }
__device__ inline float sin_theta(f3 w) { return sqrtf(sin2_theta(w)); }
__device__ inline float tan_theta(f3 w) { return sin_theta(w) / w.z; }
__device__ inline float tan2_theta(f3 w) { return sin2_theta(w) / cos2_theta(w); }
// The reference tests `sinZenith == 0` (a function name) and therefore never takes the
// zero branch (Utils/MathsCommons.h:134-143); the division is always evaluated.
__device__ inline float cos_phi(f3 w) { return clampf(w.x / sin_theta(w), -1.f, 1.f); }
__device__ inline float sin_phi(f3 w) { return clampf(w.y / sin_theta(w), -1.f, 1.f); }

// concentric disk + cosine hemisphere (Utils/RandomUtils.h:18-48)
__device__ inline f3 cosine_hemisphere(float u0, float u1) {
    float ox = 2.f * u0 - 1.f, oy = 2.f * u1 - 1.f;
    float dx = 0.f, dy = 0.f;
    if (!(ox == 0 && oy == 0)) {
        float theta, r;
        if (fabsf(ox) > fabsf(oy)) {
            r = ox;
            theta = (float)((kPiD / 4.f) * (double)(oy / ox));  // the reference's M_PI expression is double
        } else {
            r = oy;
            theta = (float)((kPiD / 2.f) - (kPiD / 4.f) * (double)(ox / oy));
        }
        dx = r * cosf(theta);
        dy = r * sinf(theta);
    }
    float z = sqrtf(fmaxf(0.f, 1 - dx * dx - dy * dy));
    return mk(dx, dy, z);
}

// ------------------------------------------------------------------------ GGX
struct GGX {
    float ax, ay;
    __device__ float D(f3 h) const {
        float t2 = tan2_theta(h);
        if (isinf(t2)) return 0;
        const float c4 = cos2_theta(h) * cos2_theta(h);
        float cp = cos_phi(h), sp = sin_phi(h);
        float e = (cp * cp / (ax * ax) + sp * sp / (ay * ay)) * t2;
        return (float)(1 / (kPiD * ax * ay * c4 * (1 + e) * (1 + e)));  // double, as M_PI makes it
    }
    __device__ float Lambda(f3 w) const {
        if (w.z == 0) return 0;
        float abs_tan = fabsf(tan_theta(w));
        float cp = cos_phi(w), sp = sin_phi(w);
        float alpha = sqrtf(cp * cp * ax * ax + sp * sp * ay * ay);
        float a2t2 = (alpha * abs_tan) * (alpha * abs_tan);
        return (-1 + sqrtf(1.f + a2t2)) / 2;
    }
    __device__ float G1(f3 w) const { return 1 / (1 + Lambda(w)); }
    __device__ float G(f3 wi, f3 wo) const { return 1.f / (1.f + Lambda(wi) + Lambda(wo)); }
    __device__ float pdf(f3 h, f3 wo) const { return D(h) * G1(wo) * fabsf(dot3(wo, h)) / fabsf(wo.z); }
    // Heitz' visible-normal sampling as in MicrofacetDistribution.h sample/sampleGGX11
    __device__ static void sample11(float cos_t, float U1, float U2, float& sx, float& sy) {
        if (cos_t > .9999) {
            float r = sqrtf(U1 / (1 - U1));
            float phi = (float)(6.28318530718 * U2);
            sx = r * cosf(phi);
            sy = r * sinf(phi);
            return;
        }
        float sin_t = sqrtf(fmaxf(0.f, 1.f - cos_t * cos_t));
        float tan_t = sin_t / cos_t;
        float a = 1 / tan_t;
        float G1v = 2 / (1 + sqrtf(1.f + 1.f / (a * a)));
        float A = 2 * U1 / G1v - 1;
        float tmp = 1.f / (A * A - 1.f);
        if (tmp > 1e10) tmp = 1e10f;
        float B = tan_t;
        float Dd = sqrtf(fmaxf(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.f));
        float s1 = B * tmp - Dd, s2 = B * tmp + Dd;
        sx = (A < 0 || s2 > 1.f / tan_t) ? s1 : s2;
        float S;
        if (U2 > 0.5f) {
            S = 1.f;
            U2 = 2.f * (U2 - .5f);
        } else {
            S = -1.f;
            U2 = 2.f * (.5f - U2);
        }
        float z = (U2 * (U2 * (U2 * 0.27385f - 0.73369f) + 0.46341f)) /
                  (U2 * (U2 * (U2 * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
        sy = S * z * sqrtf(1.f + sx * sx);
    }
    __device__ f3 sample(float u0, float u1, f3 wo) const {
        bool flip = wo.z < 0;
        if (flip) wo = neg(wo);
        f3 ws = normalize3(mk(ax * wo.x, ay * wo.y, wo.z));
        float sx, sy;
        sample11(ws.z, u0, u1, sx, sy);
        float cp = cos_phi(ws), sp = sin_phi(ws);
        float t = cp * sx - sp * sy;
        sy = sp * sx + cp * sy;
        sx = t;
        sx = ax * sx;
        sy = ay * sy;
        f3 r = normalize3(mk(-sx, -sy, 1.f));
        if (flip) r = neg(r);
        return r;
    }
};

// Schlick Fresnel (BSDFs/Fresnel.h)
__device__ inline f3 schlick(float cos_t, f3 f0) {
    float t = pow5(1 - fabsf(cos_t));
    return f0 + (mk(1, 1, 1) - f0) * t;
}

// ------------------------------------------------------------------------ BSDF
struct Bsdf {
    int type;       // pbrt material type
    f3 kd, ks, kr, kt;
    GGX ggx;
    f3 f0;          // Fresnel f0
    float eta;      // glass: aboveIOR = 1, belowIOR = eta
    float mirror;   // mirror reflectivity
    __device__ bool is_delta() const {
        return (type == cavpbrt::kGlass && !rough()) || type == cavpbrt::kMirror;
    }
    // Glass with a non-zero roughness uses MicrofacetBSDF with transmission (Materials/Glass.h)
    __device__ bool rough() const { return ggx.ax != 0.f || ggx.ay != 0.f; }

    // ---- FresnelBlend (substrate, BSDFs/Fresnel.h:65-150)
    __device__ f3 fb_eval(f3 wi, f3 wo) const {
        if (!same_hemisphere(wi, wo)) return mk(0, 0, 0);
        const f3 one = mk(1, 1, 1);
        f3 diffuse = (float)(28.f / (23.f * 3.14159265358979323846)) * kd * (one - ks) *
                     (1 - pow5(1 - .5f * fabsf(wi.z))) * (1 - pow5(1 - .5f * fabsf(wo.z)));
        f3 h = wi + wo;
        if (h.x == 0 && h.y == 0 && h.z == 0) return mk(0, 0, 0);
        h = normalize3(h);
        f3 spec = ggx.D(h) * schlick(dot3(wi, h), ks) / (4 * fabsf(dot3(wi, h)) * fmaxf(fabsf(wi.z), fabsf(wo.z)));
        return diffuse + spec;
    }
    __device__ float fb_pdf_h(f3 wi, f3 wo, f3 h) const {
        return (1.f - 0.5f) * cosine_pdf(wi.z) + 0.5f * ggx.pdf(h, wo) / (4.f * dot3(wo, h));
    }
    __device__ float fb_pdf(f3 wi, f3 wo) const { return fb_pdf_h(wi, wo, normalize3(wi + wo)); }

    // ---- microfacet transmission (rough glass, BSDFs/Microfacet.h:50-160); eta = above/below
    __device__ float mt_eta(f3 wo) const { return wo.z > 0 ? (1.f / eta) : (eta / 1.f); }
    __device__ f3 mt_eval(f3 wi, f3 wo) const {
        if (same_hemisphere(wi, wo)) return mk(0, 0, 0);
        float co = fabsf(wo.z), ci = fabsf(wi.z);
        if (ci == 0 || co == 0) return mk(0, 0, 0);
        float e = mt_eta(wo);
        f3 h = normalize3(wo + wi * e);
        if (h.z < 0) h = neg(h);
        if (dot3(wo, h) * dot3(wi, h) > 0) return mk(0, 0, 0);
        f3 F = schlick(dot3(wo, h), f0);
        float sd = dot3(wo, h) + e * dot3(wi, h);
        return (mk(1, 1, 1) - F) * kt *
               fabsf(ggx.D(h) * ggx.G(wo, wi) * e * e * fabsf(dot3(wi, h)) * fabsf(dot3(wo, h)) / (ci * co * sd * sd));
    }
    __device__ float mt_pdf(f3 wi, f3 wo) const {
        float e = mt_eta(wo);
        f3 h = normalize3(wo + wi * e);
        if (same_hemisphere(wi, wo)) return 0;
        if (dot3(wo, h) * dot3(wi, h) > 0) return 0;
        float sd = dot3(wo, h) + e * dot3(wi, h);
        float dwh = fabsf((e * e * dot3(wi, h)) / (sd * sd));
        return ggx.pdf(h, wo) * dwh;
    }
    // the reflection lobe of MicrofacetBSDF: reflectionColor kr (rough glass) or 1 (metal)
    __device__ f3 mr_eval(f3 wi, f3 wo, f3 color) const {
        if (!same_hemisphere(wi, wo)) return mk(0, 0, 0);
        float co = fabsf(wo.z), ci = fabsf(wi.z);
        f3 h = wi + wo;
        if (ci == 0 || co == 0) return mk(0, 0, 0);
        if (h.x == 0 && h.y == 0 && h.z == 0) return mk(0, 0, 0);
        h = normalize3(h);
        f3 F = schlick(dot3(wo, h), f0);
        return color * ggx.D(h) * ggx.G(wo, wi) * F / (4 * ci * co);
    }

    // ---- Lambertian
    __device__ f3 lam_eval(f3 wi, f3 wo, f3 c) const { return same_hemisphere(wi, wo) ? c / kPi : mk(0, 0, 0); }
    // ---- microfacet reflection (plastic specular)
    __device__ f3 mf_eval(f3 wi, f3 wo) const {
        if (!same_hemisphere(wi, wo)) return mk(0, 0, 0);
        float co = fabsf(wo.z), ci = fabsf(wi.z);
        f3 h = wi + wo;
        if (ci == 0 || co == 0) return mk(0, 0, 0);
        if (h.x == 0 && h.y == 0 && h.z == 0) return mk(0, 0, 0);
        h = normalize3(h);
        f3 F = schlick(dot3(wo, h), f0);
        return ks * ggx.D(h) * ggx.G(wo, wi) * F / (4 * ci * co);
    }
    __device__ float mf_pdf(f3 wi, f3 wo) const {
        f3 h = normalize3(wi + wo);
        return ggx.pdf(h, wo) / (4.f * dot3(wo, h));
    }
    // ---- specular glass (Specular.h)
    __device__ static bool refract(f3 in, f3 n, float eta, f3& out) {
        float ci = dot3(n, in);
        float s2i = fmaxf(0.f, 1.f - ci * ci);
        float s2t = eta * eta * s2i;
        if (s2t >= 1) return false;
        float ct = sqrtf(1 - s2t);
        out = eta * neg(in) + (eta * ci - ct) * n;
        return true;
    }
    __device__ float glass_reflect_prob(f3 wo) const {
        float p = schlick(fabsf(wo.z), f0).x;
        if (all_zero(kr)) p = 0;
        else if (all_zero(kt)) p = 1;
        return p;
    }

    __device__ f3 eval(f3 wi, f3 wo) const {
        switch (type) {
            case cavpbrt::kMatte: return lam_eval(wi, wo, kd);
            case cavpbrt::kPlastic: return lam_eval(wi, wo, kd) + mf_eval(wi, wo);
            case cavpbrt::kMirror:
                if (!(wi.x == -wo.x && wi.y == -wo.y && wi.z == wo.z)) return mk(0, 0, 0);
                return mk(1, 1, 1) * mirror / fabsf(wi.z);
            case cavpbrt::kMetal: return mr_eval(wi, wo, mk(1, 1, 1));
            case cavpbrt::kSubstrate: return fb_eval(wi, wo);
            case cavpbrt::kGlass: {
                if (rough()) return same_hemisphere(wi, wo) ? mr_eval(wi, wo, kr) : mt_eval(wi, wo);
                if (same_hemisphere(wi, wo)) {
                    if (!(wi.x == -wo.x && wi.y == -wo.y && wi.z == wo.z)) return mk(0, 0, 0);
                    return kr * schlick(fabsf(wi.z), f0) / fabsf(wi.z);
                }
                float e = wo.z > 0 ? (1.f / eta) : (eta / 1.f);
                f3 n = mk(0, 0, wo.z < 0 ? -1.f : 1.f);
                f3 r;
                if (!refract(wo, n, e, r)) return mk(0, 0, 0);
                if (!(r.x == wi.x && r.y == wi.y && r.z == wi.z)) return mk(0, 0, 0);
                return kt * (mk(1, 1, 1) - schlick(fabsf(wi.z), f0)) / fabsf(wi.z);
            }
        }
        return mk(0, 0, 0);
    }

    __device__ float pdf(f3 wi, f3 wo) const {
        switch (type) {
            case cavpbrt::kMatte: return cosine_pdf(wi.z);
            case cavpbrt::kPlastic: return 0.5f * cosine_pdf(wi.z) + (1.f - 0.5f) * mf_pdf(wi, wo);
            case cavpbrt::kMirror: return (wi.x == -wo.x && wi.y == -wo.y && wi.z == wo.z) ? 1.f : 0.f;
            case cavpbrt::kMetal: return mf_pdf(wi, wo);
            case cavpbrt::kSubstrate: return fb_pdf(wi, wo);
            case cavpbrt::kGlass: {
                if (rough()) {
                    const float p = glass_reflect_prob(wo);
                    return same_hemisphere(wi, wo) ? p * mf_pdf(wi, wo) : (1.f - p) * mt_pdf(wi, wo);
                }
                if (same_hemisphere(wi, wo)) {
                    if (!(wi.x == -wo.x && wi.y == -wo.y && wi.z == wo.z)) return 0;
                    return glass_reflect_prob(wo);
                }
                float e = wo.z > 0 ? (1.f / eta) : (eta / 1.f);
                f3 n = mk(0, 0, wo.z < 0 ? -1.f : 1.f);
                f3 r;
                if (!refract(wo, n, e, r)) return 0;
                if (!(r.x == wi.x && r.y == wi.y && r.z == wi.z)) return 0;
                return 1.f - glass_reflect_prob(wo);
            }
        }
        return 0;
    }

    // BSDF::sample: returns f, writes wi and pdf
    __device__ f3 sample(float u0, float u1, f3 wo, f3& wi, float& pdf_out) const {
        switch (type) {
            case cavpbrt::kMatte: {
                wi = cosine_hemisphere(u0, u1);
                pdf_out = cosine_pdf(wi.z);
                if (wo.z < 0) wi.z *= -1;
                return lam_eval(wi, wo, kd);
            }
            case cavpbrt::kPlastic: {
                if (u0 < 0.5f) {
                    u0 = u0 * (1.f / 0.5f);
                    wi = cosine_hemisphere(u0, u1);
                    if (wo.z < 0) wi.z *= -1;
                } else {
                    u0 = (u0 - 0.5f) * (1.f / (1.f - 0.5f));
                    f3 h = ggx.sample(u0, u1, wo);
                    wi = 2.0f * h * dot3(h, wo) - wo;  // reflectF
                }
                pdf_out = pdf(wi, wo);
                return eval(wi, wo);
            }
            case cavpbrt::kMirror: {
                wi = neg(wo);
                wi.z = wo.z;
                pdf_out = 1;
                return eval(wi, wo);
            }
            case cavpbrt::kMetal: {  // MicrofacetBSDF::sampleReflection: pdf from the sampled half vector
                f3 h = ggx.sample(u0, u1, wo);
                wi = 2.0f * h * dot3(h, wo) - wo;
                pdf_out = ggx.pdf(h, wo) / (4.f * dot3(wo, h));
                return mr_eval(wi, wo, mk(1, 1, 1));
            }
            case cavpbrt::kSubstrate: {  // FresnelBlendBSDF::sample
                f3 h;
                if (u0 < 0.5f) {
                    u0 = u0 * (1.f / 0.5f);
                    h = ggx.sample(u0, u1, wo);
                    wi = 2.0f * h * dot3(h, wo) - wo;
                    if (!same_hemisphere(wi, wo)) {
                        pdf_out = 0.f;  // the reference returns without setting the pdf
                        return mk(0, 0, 0);
                    }
                } else {
                    u0 = (u0 - 0.5f) * (1.f / (1.f - 0.5f));
                    wi = cosine_hemisphere(u0, u1);
                    if (wo.z < 0) wi.z *= -1;
                    h = normalize3(wi + wo);
                }
                pdf_out = fb_pdf_h(wi, wo, h);
                return fb_eval(wi, wo);
            }
            case cavpbrt::kGlass: {
                float p = glass_reflect_prob(wo);
                if (rough()) {  // MicrofacetBSDF::sample with transmission
                    if (u0 < p) {
                        u0 = u0 * (1.f / p);
                        f3 h = ggx.sample(u0, u1, wo);
                        wi = 2.0f * h * dot3(h, wo) - wo;
                        pdf_out = ggx.pdf(h, wo) / (4.f * dot3(wo, h)) * p;
                        return mr_eval(wi, wo, kr);
                    }
                    u0 = (u0 - p) * (1.f / (1.f - p));
                    f3 h = ggx.sample(u0, u1, wo);
                    if (!refract(wo, h, mt_eta(wo), wi)) {
                        pdf_out = 0.f;  // the reference returns without setting the pdf
                        return mk(0, 0, 0);
                    }
                    pdf_out = mt_pdf(wi, wo) * (1.f - p);
                    return mt_eval(wi, wo);
                }
                if (u0 < p) {
                    wi = mk(-wo.x, -wo.y, wo.z);
                    pdf_out = 1 * p;
                    return same_hemisphere(wi, wo) ? kr * schlick(fabsf(wi.z), f0) / fabsf(wi.z) : mk(0, 0, 0);
                }
                float e = wo.z > 0 ? (1.f / eta) : (eta / 1.f);
                f3 n = mk(0, 0, wo.z < 0 ? -1.f : 1.f);
                if (!refract(wo, n, e, wi)) {
                    pdf_out = 0;  // left as set before the reference's early return
                    return mk(0, 0, 0);
                }
                pdf_out = 1 * (1.f - p);
                return same_hemisphere(wi, wo) ? mk(0, 0, 0) : kt * (mk(1, 1, 1) - schlick(fabsf(wi.z), f0)) / fabsf(wi.z);
            }
        }
        pdf_out = 0;
        return mk(0, 0, 0);
    }
};

__device__ inline float mis_power(float a, float b) {
    a *= a;
    b *= b;
    return a / (a + b);
}

// ------------------------------------------------------------------------ scene
struct DevScene {
    const float* pos;       // 3 per vertex (global)
    const int32_t* idx;     // 3 per triangle (global vertex ids)
    const float* nrm;       // 3 per vertex or nullptr
    const int32_t* tri_mesh;
    const RMesh* meshes;
    const RMaterial* mats;
    const RLight* lights;
    int n_lights;
    // DirectLightingIntegrator (Integrators/DirectLightingIntegrator.cu:22-89): emission plus
    // one light sample per camera ray, without MIS weights and without a continuation
    int direct;
    const float* uv;                  // 2 per vertex, or null
    const cudaTextureObject_t* tex;   // image textures
    int env;                          // the environment light rays leaving the scene see, or -1
    // First dimension of a bounce's continuation, relative to the bounce's first: randInt +
    // rand4 + the light sample, synchronised to the maximum over the bounce's paths.  An area
    // light draws 3 (a triangle and a point; see sample_light_surface), an environment 2
    // (rand2), so 8 whenever the scene has an area light and 7 with environments only.
    int cont_dim;
    Halton halton;
};

__device__ inline Bsdf make_bsdf(const RMaterial& m) {
    Bsdf b;
    b.type = m.type;
    b.kd = ld3(m.kd);
    b.ks = ld3(m.ks);
    b.kr = ld3(m.kr);
    b.kt = ld3(m.kt);
    b.ggx = GGX{m.alpha_u, m.alpha_v};
    b.f0 = ld3(m.f0);
    b.eta = m.eta;
    b.mirror = m.mirror_kr;
    return b;
}

// Triangle normal at (u, v): Core/TriangleMesh.h getNormal / Triangle::fillIntersectionInformation
__device__ inline f3 tri_normal(const DevScene& S, const RMesh& M, int t, float u, float v) {
    int a = S.idx[3 * t], b = S.idx[3 * t + 1], c = S.idx[3 * t + 2];
    f3 n;
    if (M.has_normals) {
        f3 n0 = ld3(S.nrm + 3 * a), n1 = ld3(S.nrm + 3 * b), n2 = ld3(S.nrm + 3 * c);
        n = normalize3(n0 * (1.f - u - v) + u * n1 + v * n2);
    } else {
        f3 p0 = ld3(S.pos + 3 * a), p1 = ld3(S.pos + 3 * b), p2 = ld3(S.pos + 3 * c);
        n = normalize3(cross3(p1 - p0, p2 - p0));
    }
    if (M.reverse) n = n * -1.f;
    return n;
}

// --------------------------------------------------------------- light surfaces
struct LightPoint {
    f3 p, n;
    float pdf;  // solid-angle pdf seen from the shading point
};

// TriangleMesh::sampleSphere (Core/TriangleMesh.h:154-210): a point of the sphere inside
// the cone it subtends from `seen`, uniform in solid angle (pbrt-v3 Sphere::Sample).
__device__ inline LightPoint sample_sphere_cone(const RMesh& M, f3 seen, float u0, float u1) {
    const f3 c = mk(M.sphere[0], M.sphere[1], M.sphere[2]);
    const float radius = M.sphere[3];
    const float dc = length3(seen - c);
    const float inv_dc = 1 / dc;
    const f3 wc = (c - seen) * inv_dc;
    const Frame fr = make_frame(wc);
    const float sin_max = radius * inv_dc;
    const float sin_max2 = sin_max * sin_max;
    const float inv_sin_max = 1 / sin_max;
    const float cos_max = sqrtf(fmaxf(0.f, 1 - sin_max2));
    float cos_t = (cos_max - 1) * u0 + 1;
    float sin_t2 = 1 - cos_t * cos_t;
    if (sin_max2 < 0.00068523f) {  // sin^2(1.5 deg): series form for small cones
        sin_t2 = sin_max2 * u0;
        cos_t = sqrtf(1 - sin_t2);
    }
    const float cos_a = sin_t2 * inv_sin_max + cos_t * sqrtf(fmaxf(0.f, 1.f - sin_t2 * inv_sin_max * inv_sin_max));
    const float sin_a = sqrtf(fmaxf(0.f, 1.f - cos_a * cos_a));
    const float phi = (float)(u1 * 2 * 3.14159265358979323846);
    f3 nw = (sin_a * cosf(phi) * fr.t0 + sin_a * sinf(phi) * fr.t1 + cos_t * wc) * -1.f;
    LightPoint lp;
    lp.p = c + radius * nw;
    lp.n = M.reverse ? nw * -1.f : nw;
    lp.pdf = (float)(1 / (2 * 3.14159265358979323846 * (1 - cos_max)));
    return lp;
}

// TriangleMesh::sample (Core/TriangleMesh.h:110-152) for DiffuseAreaLight::sampleRayToPoint:
// the cone of a sphere seen from outside (2 dimensions), else a triangle picked uniformly
// and a uniform point on it (3 dimensions).  Advances `dim`.  The bounce's next draws start 8
// dimensions after its first in every case: the reference synchronises dimensions to the
// maximum over the bounce's paths, and a path that hits a tessellated light sphere shades
// from inside the true sphere and takes the 3-dimension branch.  (Only a bounce in which no
// path samples a light by triangles -- every light a sphere and no path inside one -- would
// start one dimension earlier in the reference.)
__device__ inline LightPoint sample_light_surface(const DevScene& S, const RMesh& LM, f3 seen, uint64_t index,
                                                  int& dim) {
    if (LM.shape == kShapeSphere) {
        const f3 c = mk(LM.sphere[0], LM.sphere[1], LM.sphere[2]);
        const f3 dv = seen - c;
        if (dot3(dv, dv) > LM.sphere[3] * LM.sphere[3]) {
            const float u0 = halton(S.halton, index, dim);
            const float u1 = halton(S.halton, index, dim);
            return sample_sphere_cone(LM, seen, u0, u1);
        }
    }
    const int lt = LM.first_tri + halton_int(S.halton, index, dim, LM.tri_count);
    const float temp = sqrtf(halton(S.halton, index, dim));
    const float su = 1 - temp;
    const float sv = temp * halton(S.halton, index, dim);
    const int a = S.idx[3 * lt], b = S.idx[3 * lt + 1], c = S.idx[3 * lt + 2];
    LightPoint lp;
    lp.p = ld3(S.pos + 3 * a) * su + ld3(S.pos + 3 * b) * sv + ld3(S.pos + 3 * c) * (1.f - su - sv);
    lp.n = tri_normal(S, LM, lt, su, sv);
    const f3 l2s = seen - lp.p;
    const float lcos = fabsf(dot3(lp.n, normalize3(l2s)));
    lp.pdf = dot3(l2s, l2s) / (lcos * LM.area);
    return lp;
}

// TriangleMesh::pdf (Core/TriangleMesh.h:213-232): the light pdf of a ray from `o` that
// reached the light surface at p with normal n.
__device__ inline float light_surface_pdf(const RMesh& LM, f3 o, f3 p, f3 n) {
    if (LM.shape == kShapeSphere) {
        const f3 c = mk(LM.sphere[0], LM.sphere[1], LM.sphere[2]);
        const f3 dv = o - c;
        const float d2 = dot3(dv, dv);
        const float r2 = LM.sphere[3] * LM.sphere[3];
        if (d2 > r2) {
            const float cos_max = sqrtf(fmaxf(0.f, 1.f - r2 / d2));
            return (float)(1.f / (2.f * 3.14159265358979323846 * (1 - cos_max)));
        }
    }
    const f3 l2s = o - p;
    const float cosine = fabsf(dot3(n, normalize3(l2s)));
    return dot3(l2s, l2s) / (cosine * LM.area);
}

// ------------------------------------------------------------ textures, environment
// IntersectionResult::textureCoordinates (Core/Triangle.h:128-131)
__device__ inline float2 hit_texcoord(const DevScene& S, int t, float u, float v) {
    if (!S.uv) return make_float2(0.f, 0.f);
    const int a = S.idx[3 * t], b = S.idx[3 * t + 1], c = S.idx[3 * t + 2];
    const float w = 1.f - u - v;
    return make_float2(S.uv[2 * a] * w + u * S.uv[2 * b] + v * S.uv[2 * c],
                       S.uv[2 * a + 1] * w + u * S.uv[2 * b + 1] + v * S.uv[2 * c + 1]);
}

// Material::getBSDF with a "texture Kd": the matte colour times the texel, the plastic and
// substrate diffuse colour replaced by it (Materials/{MatteMaterial,Plastic,Substrate}.h).
__device__ inline Bsdf material_bsdf(const DevScene& S, const RMaterial& m, int prim, float u, float v) {
    Bsdf b = make_bsdf(m);
    if (m.kd_tex >= 0) {
        const float2 tc = hit_texcoord(S, prim, u, v);
        const float4 tx = tex2D<float4>(S.tex[m.kd_tex], tc.x, tc.y);
        const f3 c = mk(tx.x, tx.y, tx.z);
        b.kd = m.type == cavpbrt::kMatte ? b.kd * c : c;
    }
    return b;
}

// EnvironmentMap::evaluateRay (Core/Light.h:93-113): the colour, times the texel at the
// direction's spherical coordinates in the light's frame when there is an image.
__device__ inline f3 env_eval(const DevScene& S, const RLight& L, f3 d) {
    f3 r = mk(L.L[0], L.L[1], L.L[2]);
    if (L.tex >= 0) {
        const f3 dl = mk(L.w2l[0] * d.x + L.w2l[1] * d.y + L.w2l[2] * d.z,
                         L.w2l[3] * d.x + L.w2l[4] * d.y + L.w2l[5] * d.z,
                         L.w2l[6] * d.x + L.w2l[7] * d.y + L.w2l[8] * d.z);
        float phi = atan2f(dl.y, dl.x);
        phi = (phi < 0) ? (float)(phi + 2 * 3.14159265358979323846) : phi;
        const float theta = acosf(clampf(dl.z, -1.f, 1.f));
        const float tu = (float)(phi / (2.f * 3.14159265358979323846));
        const float tv = (float)(theta / 3.14159265358979323846);
        const float4 tx = tex2D<float4>(S.tex[L.tex], tu, tv);
        r = r * mk(tx.x, tx.y, tx.z);
    }
    return r;
}

// DiffuseAreaLight / EnvironmentMap::sampleRayToPoint: direction, solid-angle pdf, incident
// radiance, and the shadow ray's length and target mesh (infinite and none for an
// environment).  Advances `dim` by 2 (environment, sphere cone) or 3 (triangle).
struct LightSample {
    f3 dir;
    float pdf;
    f3 incident;
    float dist;
    int target;
};
__device__ inline LightSample sample_light(const DevScene& S, const RLight& L, f3 pos, uint64_t index, int& dim) {
    LightSample ls;
    if (L.kind == kLightEnvironment) {
        // uniformSampleSphere (Utils/RandomUtils.h:70-78) as written: the latitude is drawn
        // uniformly, with the uniform pdf 1 / (4 pi)
        const float u0 = halton(S.halton, index, dim);
        const float u1 = halton(S.halton, index, dim);
        const float a = (float)(u0 * 2 * 3.14159265358979323846);
        const float b = (float)((u1 - 0.5) * 3.14159265358979323846);
        ls.dir = mk(cosf(b) * cosf(a), sinf(b), cosf(b) * sinf(a));
        ls.pdf = (float)(1.f / (4.f * 3.14159265358979323846));
        ls.incident = env_eval(S, L, ls.dir);
        ls.dist = INFINITY;
        ls.target = -1;
        return ls;
    }
    const RMesh& LM = S.meshes[L.mesh];
    const LightPoint lp = sample_light_surface(S, LM, pos, index, dim);
    ls.pdf = lp.pdf;
    ls.dir = normalize3(lp.p - pos);
    ls.incident = dot3(ls.dir, lp.n) >= 0 ? mk(0, 0, 0) : mk(L.L[0], L.L[1], L.L[2]);
    ls.dist = length3(lp.p - pos);
    ls.target = L.mesh;
    return ls;
}

// ---------------------------------------------------------------- path state
struct Paths {
    uint64_t* sample_index;
    float2* film_xy;
    float* result;      // 3 per path
    float* throughput;  // 3 per path
    float* mat_pdf;
    uint8_t* delta;
};

struct Queues {
    int32_t* active;      // path ids of this bounce's rays (compacted)
    cav_ray* rays;
    int32_t* next_active;
    cav_ray* next_rays;
    int32_t* hit_prim;
    float* hit_t;
    float* hit_uv;
    cav_ray* shadow_rays;
    float* shadow_limit;
    int32_t* shadow_excl;  // 2 per shadow ray
    int32_t* shadow_path;
    float* shadow_contrib; // 3 per shadow ray
    uint8_t* shadow_occ;
    uint32_t* counters;    // [0] next rays, [1] shadow rays
};

struct Camera {
    float c2w[16];
    float depth;
    int width, height;
};

__device__ inline f3 apply_pt(const float* m, f3 v) {
    float t0 = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12];
    float t1 = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13];
    float t2 = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14];
    float t3 = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15];
    return mk(t0 / t3, t1 / t3, t2 / t3);
}

// genCameraSampleSPPs (Core/Sampler.cu:29-51) + genInitialRays (PathTracingIntegrator.cu:252-266)
// dev_fc (or null): {first, count} read from device memory, for graph-replayed chunks
__global__ void k_generate(Camera cam, Halton H, int spp, int64_t first, int64_t count, Paths P, Queues Q,
                           const int64_t* dev_fc = nullptr) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (dev_fc) {
        first = dev_fc[0];
        count = dev_fc[1];
    }
    if (i >= count) return;
    int64_t s = first + i;  // global sample number, pixel-major
    int64_t pixel = s / spp;
    int x = (int)(pixel % cam.width), y = (int)(pixel / cam.width);
    uint64_t index = (uint64_t)pixel * spp + (uint64_t)(s % spp);
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

__device__ inline uint32_t warp_append(uint32_t* counter, bool pred) {
    unsigned m = __ballot_sync(0xffffffffu, pred);
    if (m == 0) return 0;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

// addSamplesToFilm + Film::addSample (Core/Film.h:26-49) with the box filter of
// Filters/BoxFilter.h ("triangle" maps to it, Filters/FilterObject.h:83-84).
__global__ void k_film(int64_t n, Paths P, int width, int height, float xw, float yw, float* sum, float* wsum,
                       const int64_t* dev_fc = nullptr) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (dev_fc) n = dev_fc[1];
    if (i >= n) return;
    f3 s = ld3(P.result + 3 * i);
    if (!finite3(s)) return;
    float2 xy = P.film_xy[i];
    int x0 = (int)floorf(xy.x - xw), x1 = (int)ceilf(xy.x + xw);
    int y0 = (int)floorf(xy.y - yw), y1 = (int)ceilf(xy.y + yw);
    for (int x = x0; x <= x1; ++x)
        for (int y = y0; y <= y1; ++y) {
            if (x >= width || y >= height || x < 0 || y < 0) continue;
            float wgt = (fabsf(x - xy.x) > xw || fabsf(y - xy.y) > yw) ? 0.f : 1.f;
            if (wgt > 0) {
                int idx = y * width + x;
                atomicAdd(sum + 3 * idx, s.x * wgt);
                atomicAdd(sum + 3 * idx + 1, s.y * wgt);
                atomicAdd(sum + 3 * idx + 2, s.z * wgt);
                atomicAdd(wsum + idx, wgt);
            }
        }
}

template <typename T>
T* carve(unsigned char*& p, size_t count) {
    size_t off = ((uintptr_t)p + 255) & ~(uintptr_t)255;
    T* r = reinterpret_cast<T*>(off);
    p = reinterpret_cast<unsigned char*>(off + sizeof(T) * count);
    return r;
}

}  // namespace
}  // namespace cav

// =================================================================== host objects
struct cav_scene {
    int device = 0;
    cavpbrt::Scene desc;
    int64_t n_tri = 0, n_vert = 0;
    float* d_pos = nullptr;
    int32_t* d_idx = nullptr;
    float* d_nrm = nullptr;
    int32_t* d_tri_mesh = nullptr;
    cav::RMesh* d_meshes = nullptr;
    cav::RMaterial* d_mats = nullptr;
    cav::RLight* d_lights = nullptr;
    float* d_uv = nullptr;                        // 2 per vertex, or null when no mesh has uvs
    std::vector<cudaArray_t> tex_arrays;          // image textures (uchar4, linear filter, wrap)
    std::vector<cudaTextureObject_t> tex_objects;
    cudaTextureObject_t* d_tex = nullptr;
    uint32_t* d_primes = nullptr;  // Halton tables: the context's (shared by its scenes)
    uint32_t* d_perm_start = nullptr;
    uint16_t* d_perms = nullptr;
    cav_bvh* bvh = nullptr;
    int bvh_rounds = 0;
    bool async_mem = false;  // arrays are stream-ordered allocations (scene_upload with async)
    cudaStream_t graph_stream = nullptr;  // private stream for graph capture and replay
    // per-stage timing of the last render: event pairs on the render stream
    struct Log {
        std::vector<cudaEvent_t> pool;
        size_t used = 0;
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> closest, shade, any;
        cudaEvent_t start = nullptr, end = nullptr;
        int64_t paths = 0, closest_rays = 0, shadow_rays = 0;
        int bounces = 0;
        bool graph = false;                      // the last render was graph-replayed
        unsigned long long* totals_h = nullptr;  // pinned: its closest / shadow ray totals
        cudaEvent_t next() {
            if (used == pool.size()) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                pool.push_back(e);
            }
            return pool[used++];
        }
        void reset() {
            used = 0;
            graph = false;
            closest.clear();
            shade.clear();
            any.clear();
            paths = closest_rays = shadow_rays = 0;
            bounces = 0;
        }
    } log;
    unsigned long long* log_totals_host() {
        if (!log.totals_h) cudaMallocHost(&log.totals_h, 16);
        return log.totals_h;
    }
};


namespace cav {
namespace {
inline DevScene dev_scene_of(const cav_scene* sc) {
    DevScene S;
    S.pos = sc->d_pos;
    S.idx = sc->d_idx;
    S.nrm = sc->d_nrm;
    S.tri_mesh = sc->d_tri_mesh;
    S.meshes = sc->d_meshes;
    S.mats = sc->d_mats;
    S.lights = sc->d_lights;
    S.n_lights = (int)sc->desc.lights.size();
    S.direct = 0;
    S.uv = sc->d_uv;
    S.tex = sc->d_tex;
    S.env = sc->desc.environment;
    S.cont_dim = 7;
    for (const auto& l : sc->desc.lights)
        if (l.kind == 0) S.cont_dim = 8;
    S.halton = Halton{sc->d_primes, sc->d_perm_start, sc->d_perms};
    return S;
}
// Film resolution of a render: the options' override, else the scene's Film.
inline void film_size(const cav_scene* sc, const cav_render_opts* o, int& w, int& h) {
    w = sc->desc.width;
    h = sc->desc.height;
    if (o && o->width > 0 && o->height > 0) {
        w = o->width;
        h = o->height;
    }
}
// PerspectiveCamera constructor (Cameras/PerspectiveCamera.cu:6-20) for a W x H film
inline Camera camera_of(const cav_scene* sc, int W, int H) {
    const cavpbrt::Scene& D = sc->desc;
    Camera cam;
    std::memcpy(cam.c2w, D.camera_to_world.data(), 64);
    cam.width = W;
    cam.height = H;
    float fov = D.fov_deg * 3.14159265358979323846f / 180.f;
    if (H <= W) cam.depth = (H / 2.f) / std::tan(fov / 2.f);
    else cam.depth = (W / 2.f) / std::tan(fov / 2.f);
    return cam;
}
}  // namespace
// guided.cu: the MLP-guided path integrator
cav_status render_guided(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                         cudaStream_t s, cav_mlp* net, const cav_guide_opts* gopt, cav_guide_stats* gstats);
// rlpath.cu: the reinforcement-learning path integrator (Q-table guided directions)
cav_status render_rlpath(cav_ctx* ctx, cav_scene* sc, const cav_render_opts* opts, float* d_sum, float* d_wsum,
                         cudaStream_t s);
}  // namespace cav
