/*
 * Path-tracing oracle — TEST INFRASTRUCTURE, not part of the product.
 *
 * A scalar CPU restatement of the reference's plain path integrator, one path at a time,
 * over the BVH oracle's single-ray queries (cav_oracle.c).  Only tests/ and bench.py's
 * CPU-baseline leg load it, as the checker or the timed CPU baseline.
 *
 * Reference files followed (paths inside AmesingFlank/Cavalry):
 *   Core/Sampler.cu:29-51              genCameraSampleSPPs (index, jitter dims 0/1; the stored
 *                                      state keeps dimension 0)          -> orc_render_path
 *   Cameras/PerspectiveCamera.h:33-49  genRay                             -> camera_ray
 *   Cameras/PerspectiveCamera.cu:6-20  depthForUnitSizePixel              -> orc_render_path
 *   Samplers/HaltonSampler.h:13-76     runHalton / rand1 / randInt        -> halton, halton_int
 *   Samplers/HaltonSampler.cu:7-67     primes, srand(533799) Fisher-Yates -> orc_halton_tables
 *   Integrators/PathTracingIntegrator.cu:95-249
 *                                      intersectScene / computeLighting / evalMaterial /
 *                                      genNextRay                         -> trace_path
 *   Core/Material.h:21-26              Material::eval (Li f |cos|)
 *   Lights/DiffuseAreaLight.h:26-62    sampleRayToPoint / evaluateRay / pdf
 *   Core/TriangleMesh.h:110-153, :219-225  TriangleMesh::sample / pdf
 *   Core/TriangleMesh.cu:189-199       surface area (float sum of half cross lengths)
 *   Core/IntersectionResult.h:22-52, Utils/MathsCommons.h:194-202  local frame
 *   BSDFs/Lambertian.h, PlasticBSDF.h, Microfacet.h (reflection), MicrofacetDistribution.h,
 *   Fresnel.h (Schlick), Specular.h, MirrorBSDF.h; Utils/RandomUtils.h:18-41
 *   Core/Film.h:26-49, Filters/BoxFilter.h  box splat
 *
 * Numerics.  IEEE float on the host; the reference's device build uses approximate
 * division, reciprocal, sqrt and trig instructions.  Where the reference evaluates an
 * expression in double (M_PI products, 1/double), this file does too.  A float film from
 * this oracle therefore agrees with the GPU's per pixel within rounding, except where a
 * rounding difference flips a discrete choice (a Russian-roulette or BSDF-lobe threshold,
 * a near-tie hit); the tests state the tolerance.  A path whose throughput becomes exactly
 * zero is ended, as the product does (the reference traces it on, adding only zeros).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    float bmin[3];
    float bmax[3];
    int32_t begin, end, left, right, parent, is_leaf;
    float area, cost;
} ONode;

int32_t orc_closest_one(const ONode* nodes, const float* pos, const int32_t* idx, const float* o, const float* d,
                        float* t_out, float* u_out, float* v_out);
int orc_any_one(const ONode* nodes, const float* pos, const int32_t* idx, const int32_t* mesh_of_tri,
                const float* o, const float* d, float limit, int32_t src, int32_t dst);

/* Scene records, the same field order as the product's device records. */
typedef struct {
    int32_t first_tri, tri_count, has_normals, reverse, material, light;
    float area;
    int32_t shape;    /* 0 triangle mesh, 1 tessellated sphere (cone-sampled as a light), 2 disk */
    float sphere[4];  /* sphere: world centre and radius (TriangleMesh::shapeParams) */
} OMesh;
typedef struct {
    int32_t type; /* 0 matte, 1 mirror, 2 substrate, 3 metal, 4 glass (specular or rough), 5 plastic */
    float kd[3], ks[3], kr[3], kt[3];
    float alpha_u, alpha_v, eta, mirror_kr;
    float f0[3];     /* metal: Fresnel f0 (complex IOR or copper) */
    int32_t has_f0;
    int32_t kd_tex;  /* "texture Kd": texture index, or -1 */
} OMaterial;
typedef struct {
    float L[3];
    int32_t mesh;  /* area light: its mesh */
    int32_t kind;  /* 0 area, 1 environment */
    int32_t tex;   /* environment image, or -1 */
    float w2l[9];  /* environment: mat3(worldToLight), row-major */
} OLight;
typedef struct {
    int32_t width, height;
    const uint8_t* rgba; /* 8-bit images: rows bottom-up (after the load flip), before the inverse gamma */
    const float* rgbaf;  /* OpenEXR images (when not NULL): RGBA floats, rows as stored (no flip, no gamma) */
} OTexture;

enum { M_MATTE = 0, M_MIRROR = 1, M_SUBSTRATE = 2, M_METAL = 3, M_GLASS = 4, M_PLASTIC = 5 };

/* ------------------------------------------------------------------ vectors */
typedef struct { float x, y, z; } V3;
static V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static V3 vs(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 vdivs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 vcross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static V3 vnorm(V3 a) { return vs(a, 1.0f / sqrtf(vdot(a, a))); }
static int vzero(V3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
static V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

/* ------------------------------------------------------------------ Halton */
typedef struct {
    uint32_t primes[1024];
    uint32_t start[1024];
    uint16_t* perms;
} Halton;

/* computePrimes(1024) + buildPermutations (HaltonSampler.cu:7-67): the C library's rand()
 * after srand(533799), one Fisher-Yates shuffle per prime.  Writes primes, starts and the
 * concatenated permutations (perms may be NULL to query the total length). */
int64_t orc_halton_tables(uint32_t* primes, uint32_t* start, uint16_t* perms) {
    uint32_t pr[1024];
    int np = 0;
    pr[np++] = 2;
    for (uint32_t i = 3; np < 1024; ++i) {
        int is_prime = 1;
        for (int k = 0; k < np; ++k) {
            if (pr[k] * pr[k] > i) break;
            if (i % pr[k] == 0) { is_prime = 0; break; }
        }
        if (is_prime) pr[np++] = i;
    }
    int64_t size = 0;
    for (int k = 0; k < 1024; ++k) {
        if (primes) primes[k] = pr[k];
        if (start) start[k] = (uint32_t)size;
        size += pr[k];
    }
    if (!perms) return size;
    srand(533799);
    for (int k = 0; k < 1024; ++k) {
        uint16_t* v = perms + (start ? start[k] : 0);
        for (uint32_t j = 0; j < pr[k]; ++j) v[j] = (uint16_t)j;
        for (int m = (int)pr[k] - 1; m > 0; --m) {
            int r = rand() % (m + 1);
            uint16_t t = v[m];
            v[m] = v[r];
            v[r] = t;
        }
    }
    return size;
}

static float halton(const Halton* h, uint64_t index, int* dim) {
    int d = *dim;
    *dim += 1;
    uint32_t base = h->primes[d];
    const uint16_t* perm = h->perms + h->start[d];
    float r = 0, f = 1;
    uint64_t i = index;
    while (i > 0) {
        f = f / (float)base;
        r = r + f * (float)perm[i % base];
        i = i / base;
    }
    return r;
}
static int halton_int(const Halton* h, uint64_t index, int* dim, int n) {
    float f = halton(h, index, dim);
    int r = (int)(f * (float)n);
    if (r >= n) r = n - 1;
    return r;
}

/* ------------------------------------------------------------------ frame */
typedef struct { V3 t0, t1, n; } Frame;
static Frame make_frame(V3 n) {
    Frame fr;
    fr.t0 = fabsf(n.x) < 0.5f ? vcross(v3(1, 0, 0), n) : vcross(v3(0, 1, 0), n);
    fr.t0 = vnorm(fr.t0);
    fr.t1 = vnorm(vcross(n, fr.t0));
    fr.n = n;
    return fr;
}
static V3 to_local(const Frame* f, V3 v) { return v3(vdot(f->t0, v), vdot(f->t1, v), vdot(f->n, v)); }
static V3 to_world(const Frame* f, V3 v) { return vadd(vadd(vs(f->t0, v.x), vs(f->t1, v.y)), vs(f->n, v.z)); }

/* ------------------------------------------------------------------ sampling maths */
static float clampf(float x, float lo, float hi) { return fmaxf(lo, fminf(x, hi)); }
static float cos2t(V3 w) { return w.z * w.z; }
static float sin2t(V3 w) { return fmaxf(0.f, 1.f - cos2t(w)); }
static float sint(V3 w) { return sqrtf(sin2t(w)); }
static float tant(V3 w) { return sint(w) / w.z; }
static float tan2t(V3 w) { return sin2t(w) / cos2t(w); }
/* Utils/MathsCommons.h:134-143: the zero test compares a function name, so the division
 * always runs */
static float cosp(V3 w) { return clampf(w.x / sint(w), -1.f, 1.f); }
static float sinp(V3 w) { return clampf(w.y / sint(w), -1.f, 1.f); }
static float pow5f(float f) { return (f * f) * (f * f) * f; }

static V3 cosine_hemisphere(float u0, float u1) {
    float ox = 2.f * u0 - 1.f, oy = 2.f * u1 - 1.f;
    float dx = 0, dy = 0;
    if (!(ox == 0 && oy == 0)) {
        float theta, r;
        if (fabsf(ox) > fabsf(oy)) {
            r = ox;
            theta = (float)((M_PI / 4.f) * (double)(oy / ox));
        } else {
            r = oy;
            theta = (float)((M_PI / 2.f) - (M_PI / 4.f) * (double)(ox / oy));
        }
        dx = r * cosf(theta);
        dy = r * sinf(theta);
    }
    return v3(dx, dy, sqrtf(fmaxf(0.f, 1 - dx * dx - dy * dy)));
}
static float cosine_pdf(V3 w) { return (float)fabs((double)w.z / M_PI); }

typedef struct { float ax, ay; } GGX;
static float ggx_D(GGX g, V3 h) {
    float t2 = tan2t(h);
    if (isinf(t2)) return 0;
    float c4 = cos2t(h) * cos2t(h);
    float cp = cosp(h), sp = sinp(h);
    float e = (cp * cp / (g.ax * g.ax) + sp * sp / (g.ay * g.ay)) * t2;
    return (float)(1 / (M_PI * g.ax * g.ay * c4 * (1 + e) * (1 + e)));
}
static float ggx_lambda(GGX g, V3 w) {
    if (w.z == 0) return 0;
    float at = fabsf(tant(w));
    float cp = cosp(w), sp = sinp(w);
    float alpha = sqrtf(cp * cp * g.ax * g.ax + sp * sp * g.ay * g.ay);
    float a2t2 = (alpha * at) * (alpha * at);
    return (-1 + sqrtf(1.f + a2t2)) / 2;
}
static float ggx_G1(GGX g, V3 w) { return 1 / (1 + ggx_lambda(g, w)); }
static float ggx_G(GGX g, V3 wi, V3 wo) { return 1.f / (1.f + ggx_lambda(g, wi) + ggx_lambda(g, wo)); }
static float ggx_pdf(GGX g, V3 h, V3 wo) { return ggx_D(g, h) * ggx_G1(g, wo) * fabsf(vdot(wo, h)) / fabsf(wo.z); }
static void ggx_sample11(float cos_t, float U1, float U2, float* sx, float* sy) {
    if (cos_t > .9999) {
        float r = sqrtf(U1 / (1 - U1));
        float phi = (float)(6.28318530718 * U2);
        *sx = r * cosf(phi);
        *sy = r * sinf(phi);
        return;
    }
    float sin_t = sqrtf(fmaxf(0.f, 1.f - cos_t * cos_t));
    float tan_t = sin_t / cos_t;
    float a = 1 / tan_t;
    float G1 = 2 / (1 + sqrtf(1.f + 1.f / (a * a)));
    float A = 2 * U1 / G1 - 1;
    float tmp = 1.f / (A * A - 1.f);
    if (tmp > 1e10) tmp = 1e10f;
    float B = tan_t;
    float D = sqrtf(fmaxf(B * B * tmp * tmp - (A * A - B * B) * tmp, 0.f));
    float s1 = B * tmp - D, s2 = B * tmp + D;
    *sx = (A < 0 || s2 > 1.f / tan_t) ? s1 : s2;
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
    *sy = S * z * sqrtf(1.f + *sx * *sx);
}
static V3 ggx_sample(GGX g, float u0, float u1, V3 wo) {
    int flip = wo.z < 0;
    if (flip) wo = vs(wo, -1.f);
    V3 ws = vnorm(v3(g.ax * wo.x, g.ay * wo.y, wo.z));
    float sx, sy;
    ggx_sample11(ws.z, u0, u1, &sx, &sy);
    float cp = cosp(ws), sp = sinp(ws);
    float t = cp * sx - sp * sy;
    sy = sp * sx + cp * sy;
    sx = t;
    sx = g.ax * sx;
    sy = g.ay * sy;
    V3 r = vnorm(v3(-sx, -sy, 1.f));
    if (flip) r = vs(r, -1.f);
    return r;
}
static V3 schlick(float c, V3 f0) {
    float t = pow5f(1 - fabsf(c));
    return vadd(f0, vs(vsub(v3(1, 1, 1), f0), t));
}

/* ------------------------------------------------------------------ BSDF */
typedef struct {
    int type;
    V3 kd, ks, kr, kt, f0;
    GGX g;
    float eta, mirror;
} Bsdf;

static Bsdf make_bsdf(const OMaterial* m) {
    Bsdf b;
    b.type = m->type;
    b.kd = ld3(m->kd);
    b.ks = ld3(m->ks);
    b.kr = ld3(m->kr);
    b.kt = ld3(m->kt);
    b.g.ax = m->alpha_u;
    b.g.ay = m->alpha_v;
    V3 e = v3(m->eta, m->eta, m->eta);
    V3 t = v3((e.x - 1) / (e.x + 1), (e.y - 1) / (e.y + 1), (e.z - 1) / (e.z + 1));
    b.f0 = m->has_f0 ? ld3(m->f0) : vmul(t, t);
    b.eta = m->eta;
    b.mirror = m->mirror_kr;
    return b;
}
static int same_hemi(V3 a, V3 b) { return a.z * b.z > 0; }
static int is_mirror_dir(V3 wi, V3 wo) { return wi.x == -wo.x && wi.y == -wo.y && wi.z == wo.z; }
static V3 lam_eval(V3 wi, V3 wo, V3 c) { return same_hemi(wi, wo) ? vdivs(c, (float)M_PI) : v3(0, 0, 0); }
static V3 mf_eval(const Bsdf* b, V3 wi, V3 wo) {
    if (!same_hemi(wi, wo)) return v3(0, 0, 0);
    float co = fabsf(wo.z), ci = fabsf(wi.z);
    V3 h = vadd(wi, wo);
    if (ci == 0 || co == 0) return v3(0, 0, 0);
    if (vzero(h)) return v3(0, 0, 0);
    h = vnorm(h);
    V3 F = schlick(vdot(wo, h), b->f0);
    return vdivs(vmul(vs(vs(b->ks, ggx_D(b->g, h)), ggx_G(b->g, wo, wi)), F), 4 * ci * co);
}
static float mf_pdf(const Bsdf* b, V3 wi, V3 wo) {
    V3 h = vnorm(vadd(wi, wo));
    return ggx_pdf(b->g, h, wo) / (4.f * vdot(wo, h));
}
static int refract_dir(V3 in, V3 n, float eta, V3* out) {
    float ci = vdot(n, in);
    float s2i = fmaxf(0.f, 1.f - ci * ci);
    float s2t = eta * eta * s2i;
    if (s2t >= 1) return 0;
    float ct = sqrtf(1 - s2t);
    *out = vadd(vs(vs(in, -1.f), eta), vs(n, eta * ci - ct));
    return 1;
}
static float glass_reflect_prob(const Bsdf* b, V3 wo) {
    float p = schlick(fabsf(wo.z), b->f0).x;
    if (vzero(b->kr)) p = 0;
    else if (vzero(b->kt)) p = 1;
    return p;
}
static int rough(const Bsdf* b) { return b->g.ax != 0.f || b->g.ay != 0.f; }
/* MicrofacetBSDF reflection lobe (BSDFs/Microfacet.h:25-40) with the given reflection colour */
static V3 mr_eval(const Bsdf* b, V3 wi, V3 wo, V3 color) {
    if (!same_hemi(wi, wo)) return v3(0, 0, 0);
    float co = fabsf(wo.z), ci = fabsf(wi.z);
    V3 h = vadd(wi, wo);
    if (ci == 0 || co == 0) return v3(0, 0, 0);
    if (vzero(h)) return v3(0, 0, 0);
    h = vnorm(h);
    V3 F = schlick(vdot(wo, h), b->f0);
    return vdivs(vmul(vs(vs(color, ggx_D(b->g, h)), ggx_G(b->g, wo, wi)), F), 4 * ci * co);
}
static float mt_eta(const Bsdf* b, V3 wo) { return wo.z > 0 ? (1.f / b->eta) : (b->eta / 1.f); }
/* MicrofacetBSDF transmission (BSDFs/Microfacet.h:42-62, :118-150) */
static V3 mt_eval(const Bsdf* b, V3 wi, V3 wo) {
    if (same_hemi(wi, wo)) return v3(0, 0, 0);
    float co = fabsf(wo.z), ci = fabsf(wi.z);
    if (ci == 0 || co == 0) return v3(0, 0, 0);
    float e = mt_eta(b, wo);
    V3 h = vnorm(vadd(wo, vs(wi, e)));
    if (h.z < 0) h = vs(h, -1.f);
    if (vdot(wo, h) * vdot(wi, h) > 0) return v3(0, 0, 0);
    V3 F = schlick(vdot(wo, h), b->f0);
    float sd = vdot(wo, h) + e * vdot(wi, h);
    float m = fabsf(ggx_D(b->g, h) * ggx_G(b->g, wo, wi) * e * e * fabsf(vdot(wi, h)) * fabsf(vdot(wo, h)) /
                    (ci * co * sd * sd));
    return vs(vmul(vsub(v3(1, 1, 1), F), b->kt), m);
}
static float mt_pdf(const Bsdf* b, V3 wi, V3 wo) {
    float e = mt_eta(b, wo);
    V3 h = vnorm(vadd(wo, vs(wi, e)));
    if (same_hemi(wi, wo)) return 0;
    if (vdot(wo, h) * vdot(wi, h) > 0) return 0;
    float sd = vdot(wo, h) + e * vdot(wi, h);
    return ggx_pdf(b->g, h, wo) * fabsf((e * e * vdot(wi, h)) / (sd * sd));
}
/* FresnelBlendBSDF (BSDFs/Fresnel.h:65-150) */
static V3 fb_eval(const Bsdf* b, V3 wi, V3 wo) {
    if (!same_hemi(wi, wo)) return v3(0, 0, 0);
    V3 one = v3(1, 1, 1);
    V3 diffuse = vs(vs(vmul(vs(b->kd, (float)(28.f / (23.f * M_PI))), vsub(one, b->ks)),
                       1 - pow5f(1 - .5f * fabsf(wi.z))),
                    1 - pow5f(1 - .5f * fabsf(wo.z)));
    V3 h = vadd(wi, wo);
    if (vzero(h)) return v3(0, 0, 0);
    h = vnorm(h);
    V3 spec = vdivs(vs(schlick(vdot(wi, h), b->ks), ggx_D(b->g, h)),
                    4 * fabsf(vdot(wi, h)) * fmaxf(fabsf(wi.z), fabsf(wo.z)));
    return vadd(diffuse, spec);
}
static float fb_pdf_h(const Bsdf* b, V3 wi, V3 wo, V3 h) {
    return (1.f - 0.5f) * cosine_pdf(wi) + 0.5f * ggx_pdf(b->g, h, wo) / (4.f * vdot(wo, h));
}

static V3 bsdf_eval(const Bsdf* b, V3 wi, V3 wo) {
    switch (b->type) {
        case M_MATTE: return lam_eval(wi, wo, b->kd);
        case M_PLASTIC: return vadd(lam_eval(wi, wo, b->kd), mf_eval(b, wi, wo));
        case M_MIRROR:
            if (!is_mirror_dir(wi, wo)) return v3(0, 0, 0);
            return vdivs(vs(v3(1, 1, 1), b->mirror), fabsf(wi.z));
        case M_METAL: return mr_eval(b, wi, wo, v3(1, 1, 1));
        case M_SUBSTRATE: return fb_eval(b, wi, wo);
        case M_GLASS: {
            if (rough(b)) return same_hemi(wi, wo) ? mr_eval(b, wi, wo, b->kr) : mt_eval(b, wi, wo);
            if (same_hemi(wi, wo)) {
                if (!is_mirror_dir(wi, wo)) return v3(0, 0, 0);
                return vdivs(vmul(b->kr, schlick(fabsf(wi.z), b->f0)), fabsf(wi.z));
            }
            float e = wo.z > 0 ? (1.f / b->eta) : (b->eta / 1.f);
            V3 n = v3(0, 0, wo.z < 0 ? -1.f : 1.f), r;
            if (!refract_dir(wo, n, e, &r)) return v3(0, 0, 0);
            if (!(r.x == wi.x && r.y == wi.y && r.z == wi.z)) return v3(0, 0, 0);
            return vdivs(vmul(b->kt, vsub(v3(1, 1, 1), schlick(fabsf(wi.z), b->f0))), fabsf(wi.z));
        }
    }
    return v3(0, 0, 0);
}
static float bsdf_pdf(const Bsdf* b, V3 wi, V3 wo) {
    switch (b->type) {
        case M_MATTE: return cosine_pdf(wi);
        case M_PLASTIC: return 0.5f * cosine_pdf(wi) + (1.f - 0.5f) * mf_pdf(b, wi, wo);
        case M_MIRROR: return is_mirror_dir(wi, wo) ? 1.f : 0.f;
        case M_METAL: return mf_pdf(b, wi, wo);
        case M_SUBSTRATE: return fb_pdf_h(b, wi, wo, vnorm(vadd(wi, wo)));
        case M_GLASS: {
            if (rough(b)) {
                float p = glass_reflect_prob(b, wo);
                return same_hemi(wi, wo) ? p * mf_pdf(b, wi, wo) : (1.f - p) * mt_pdf(b, wi, wo);
            }
            if (same_hemi(wi, wo)) return is_mirror_dir(wi, wo) ? glass_reflect_prob(b, wo) : 0.f;
            float e = wo.z > 0 ? (1.f / b->eta) : (b->eta / 1.f);
            V3 n = v3(0, 0, wo.z < 0 ? -1.f : 1.f), r;
            if (!refract_dir(wo, n, e, &r)) return 0;
            if (!(r.x == wi.x && r.y == wi.y && r.z == wi.z)) return 0;
            return 1.f - glass_reflect_prob(b, wo);
        }
    }
    return 0;
}
static V3 bsdf_sample(const Bsdf* b, float u0, float u1, V3 wo, V3* wi, float* pdf) {
    switch (b->type) {
        case M_MATTE:
            *wi = cosine_hemisphere(u0, u1);
            *pdf = cosine_pdf(*wi);
            if (wo.z < 0) wi->z *= -1;
            return lam_eval(*wi, wo, b->kd);
        case M_PLASTIC:
            if (u0 < 0.5f) {
                u0 = u0 * (1.f / 0.5f);
                *wi = cosine_hemisphere(u0, u1);
                if (wo.z < 0) wi->z *= -1;
            } else {
                u0 = (u0 - 0.5f) * (1.f / (1.f - 0.5f));
                V3 h = ggx_sample(b->g, u0, u1, wo);
                *wi = vsub(vs(vs(h, 2.0f), vdot(h, wo)), wo);
            }
            *pdf = bsdf_pdf(b, *wi, wo);
            return bsdf_eval(b, *wi, wo);
        case M_MIRROR:
            *wi = vs(wo, -1.f);
            wi->z = wo.z;
            *pdf = 1;
            return bsdf_eval(b, *wi, wo);
        case M_METAL: {
            V3 h = ggx_sample(b->g, u0, u1, wo);
            *wi = vsub(vs(vs(h, 2.0f), vdot(h, wo)), wo);
            *pdf = ggx_pdf(b->g, h, wo) / (4.f * vdot(wo, h));
            return mr_eval(b, *wi, wo, v3(1, 1, 1));
        }
        case M_SUBSTRATE: {
            V3 h;
            if (u0 < 0.5f) {
                u0 = u0 * (1.f / 0.5f);
                h = ggx_sample(b->g, u0, u1, wo);
                *wi = vsub(vs(vs(h, 2.0f), vdot(h, wo)), wo);
                if (!same_hemi(*wi, wo)) {
                    *pdf = 0;
                    return v3(0, 0, 0);
                }
            } else {
                u0 = (u0 - 0.5f) * (1.f / (1.f - 0.5f));
                *wi = cosine_hemisphere(u0, u1);
                if (wo.z < 0) wi->z *= -1;
                h = vnorm(vadd(*wi, wo));
            }
            *pdf = fb_pdf_h(b, *wi, wo, h);
            return fb_eval(b, *wi, wo);
        }
        case M_GLASS: {
            float p = glass_reflect_prob(b, wo);
            if (rough(b)) {
                if (u0 < p) {
                    u0 = u0 * (1.f / p);
                    V3 h = ggx_sample(b->g, u0, u1, wo);
                    *wi = vsub(vs(vs(h, 2.0f), vdot(h, wo)), wo);
                    *pdf = ggx_pdf(b->g, h, wo) / (4.f * vdot(wo, h)) * p;
                    return mr_eval(b, *wi, wo, b->kr);
                }
                u0 = (u0 - p) * (1.f / (1.f - p));
                V3 h = ggx_sample(b->g, u0, u1, wo);
                if (!refract_dir(wo, h, mt_eta(b, wo), wi)) {
                    *pdf = 0;
                    return v3(0, 0, 0);
                }
                *pdf = mt_pdf(b, *wi, wo) * (1.f - p);
                return mt_eval(b, *wi, wo);
            }
            if (u0 < p) {
                *wi = v3(-wo.x, -wo.y, wo.z);
                *pdf = 1 * p;
                return same_hemi(*wi, wo) ? vdivs(vmul(b->kr, schlick(fabsf(wi->z), b->f0)), fabsf(wi->z))
                                          : v3(0, 0, 0);
            }
            float e = wo.z > 0 ? (1.f / b->eta) : (b->eta / 1.f);
            V3 n = v3(0, 0, wo.z < 0 ? -1.f : 1.f);
            if (!refract_dir(wo, n, e, wi)) {
                *pdf = 0;
                return v3(0, 0, 0);
            }
            *pdf = 1 * (1.f - p);
            return same_hemi(*wi, wo) ? v3(0, 0, 0)
                                      : vdivs(vmul(b->kt, vsub(v3(1, 1, 1), schlick(fabsf(wi->z), b->f0))), fabsf(wi->z));
        }
    }
    *pdf = 0;
    return v3(0, 0, 0);
}
static int bsdf_delta(const Bsdf* b) { return (b->type == M_GLASS && !rough(b)) || b->type == M_MIRROR; }
static float mis_power(float a, float b) {
    a *= a;
    b *= b;
    return a / (a + b);
}

/* ------------------------------------------------------------------ scene */
typedef struct {
    const ONode* nodes;
    const float* pos;
    const int32_t* idx;
    const float* nrm;
    const int32_t* tri_mesh;
    const OMesh* meshes;
    const OMaterial* mats;
    const OLight* lights;
    int n_lights;
    int direct; /* DirectLightingIntegrator.cu:22-89: one light sample, no MIS, no continuation */
    const float* uv;            /* 2 per vertex, or NULL */
    const OTexture* textures;   /* texels after the reference's load-time inverse gamma */
    int env;                    /* environment light index, or -1 */
    int cont_dim;               /* 8 with an area light, 7 with environments only */
    Halton h;
} Scene;

static V3 tri_normal(const Scene* S, const OMesh* M, int t, float u, float v) {
    int a = S->idx[3 * t], b = S->idx[3 * t + 1], c = S->idx[3 * t + 2];
    V3 n;
    if (M->has_normals) {
        V3 n0 = ld3(S->nrm + 3 * a), n1 = ld3(S->nrm + 3 * b), n2 = ld3(S->nrm + 3 * c);
        n = vnorm(vadd(vadd(vs(n0, 1.f - u - v), vs(n1, u)), vs(n2, v)));
    } else {
        V3 p0 = ld3(S->pos + 3 * a), p1 = ld3(S->pos + 3 * b), p2 = ld3(S->pos + 3 * c);
        n = vnorm(vcross(vsub(p1, p0), vsub(p2, p0)));
    }
    if (M->reverse) n = vs(n, -1.f);
    return n;
}

static V3 apply_pt(const float* m, V3 v) {
    float t0 = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12];
    float t1 = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13];
    float t2 = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14];
    float t3 = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15];
    return v3(t0 / t3, t1 / t3, t2 / t3);
}

/* ------------------------------------------------------------------ textures */
/* Color.h inverseGammaCorrect, applied per channel at load and truncated to 8 bits
 * (Core/Texture.cu:61-68, .png files) */
static float inverse_gamma(float value) {
    if (value <= 0.04045f) return value * 1.f / 12.92f;
    return powf((value + 0.055f) * 1.f / 1.055f, (float)2.4f);
}
static uint8_t load_gamma(uint8_t c) { return (uint8_t)(255.f * inverse_gamma(c / 255.f)); }

/* The 256-entry table of load_gamma (Core/Texture.cu:19, :64-71: .png channels at load time). */
void orc_load_gamma_table(uint8_t* out) {
    for (int c = 0; c < 256; ++c) out[c] = load_gamma((uint8_t)c);
}

/* tex2D of a uchar4 texture read as normalized floats (or of a float4 texture read as it
 * is) with bilinear filtering and wrapped normalized coordinates, restated from the CUDA
 * programming guide's description of texture fetching: x = frac(u) * W - 0.5, texels
 * i = floor(x) and i + 1 (wrapped), weight frac(x) held with 8 fractional bits; the same
 * in y. */
static V3 tex_read(const OTexture* t, float u, float v) {
    float xs = (u - floorf(u)) * t->width - 0.5f, ys = (v - floorf(v)) * t->height - 0.5f;
    float fx = floorf(xs), fy = floorf(ys);
    float a = rintf((xs - fx) * 256.f) / 256.f, b = rintf((ys - fy) * 256.f) / 256.f;
    int i0 = (int)fx, j0 = (int)fy;
    V3 acc = v3(0, 0, 0);
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
            int i = ((i0 + di) % t->width + t->width) % t->width;
            int j = ((j0 + dj) % t->height + t->height) % t->height;
            float w = (di ? a : 1.f - a) * (dj ? b : 1.f - b);
            if (t->rgbaf) {
                const float* q = t->rgbaf + 4 * ((size_t)j * t->width + i);
                acc = vadd(acc, vs(v3(q[0], q[1], q[2]), w));
            } else {
                const uint8_t* p = t->rgba + 4 * ((size_t)j * t->width + i);
                acc = vadd(acc, vs(v3(load_gamma(p[0]) / 255.f, load_gamma(p[1]) / 255.f, load_gamma(p[2]) / 255.f), w));
            }
        }
    return acc;
}

/* IntersectionResult::textureCoordinates (Core/Triangle.h:128-131) */
static void hit_texcoord(const Scene* S, int t, float u, float v, float* tu, float* tv) {
    if (!S->uv) {
        *tu = *tv = 0.f;
        return;
    }
    int a = S->idx[3 * t], b = S->idx[3 * t + 1], c = S->idx[3 * t + 2];
    float w = 1.f - u - v;
    *tu = S->uv[2 * a] * w + u * S->uv[2 * b] + v * S->uv[2 * c];
    *tv = S->uv[2 * a + 1] * w + u * S->uv[2 * b + 1] + v * S->uv[2 * c + 1];
}

/* EnvironmentMap::evaluateRay (Core/Light.h:93-113) */
static V3 env_eval(const Scene* S, const OLight* L, V3 d) {
    V3 r = ld3(L->L);
    if (L->tex >= 0) {
        const float* m = L->w2l;
        V3 dl = v3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[3] * d.x + m[4] * d.y + m[5] * d.z,
                   m[6] * d.x + m[7] * d.y + m[8] * d.z);
        float phi = atan2f(dl.y, dl.x);
        phi = (phi < 0) ? (float)(phi + 2 * M_PI) : phi;
        float theta = acosf(fminf(fmaxf(dl.z, -1.f), 1.f));
        V3 tx = tex_read(&S->textures[L->tex], (float)(phi / (2.f * M_PI)), (float)(theta / M_PI));
        r = vmul(r, tx);
    }
    return r;
}

/* TriangleMesh::sampleSphere (Core/TriangleMesh.h:154-210): uniform in the cone a sphere
 * subtends from `seen` (pbrt-v3 Sphere::Sample), solid-angle pdf. */
static void sphere_cone(const OMesh* M, V3 seen, float u0, float u1, V3* lp, V3* ln, float* pdf) {
    V3 c = v3(M->sphere[0], M->sphere[1], M->sphere[2]);
    float radius = M->sphere[3];
    V3 dv = vsub(seen, c);
    float dc = sqrtf(vdot(dv, dv));
    float inv_dc = 1 / dc;
    V3 wc = vs(vsub(c, seen), inv_dc);
    Frame fr = make_frame(wc);
    float sin_max = radius * inv_dc;
    float sin_max2 = sin_max * sin_max;
    float inv_sin_max = 1 / sin_max;
    float cos_max = sqrtf(fmaxf(0.f, 1 - sin_max2));
    float cos_t = (cos_max - 1) * u0 + 1;
    float sin_t2 = 1 - cos_t * cos_t;
    if (sin_max2 < 0.00068523f) {
        sin_t2 = sin_max2 * u0;
        cos_t = sqrtf(1 - sin_t2);
    }
    float cos_a = sin_t2 * inv_sin_max + cos_t * sqrtf(fmaxf(0.f, 1.f - sin_t2 * inv_sin_max * inv_sin_max));
    float sin_a = sqrtf(fmaxf(0.f, 1.f - cos_a * cos_a));
    float phi = (float)(u1 * 2 * M_PI);
    V3 nw = vs(vadd(vadd(vs(fr.t0, sin_a * cosf(phi)), vs(fr.t1, sin_a * sinf(phi))), vs(wc, cos_t)), -1.f);
    *lp = vadd(c, vs(nw, radius));
    *ln = M->reverse ? vs(nw, -1.f) : nw;
    *pdf = (float)(1 / (2 * M_PI * (1 - cos_max)));
}

/* TriangleMesh::sample (Core/TriangleMesh.h:110-152): the sphere cone seen from outside (2
 * dimensions), else a uniform triangle and a uniform point on it (3 dimensions). */
static void light_sample(const Scene* S, const OMesh* LM, V3 seen, uint64_t index, int* dim, V3* lp, V3* ln,
                         float* pdf) {
    if (LM->shape == 1) {
        V3 dv = vsub(seen, v3(LM->sphere[0], LM->sphere[1], LM->sphere[2]));
        if (vdot(dv, dv) > LM->sphere[3] * LM->sphere[3]) {
            float u0 = halton(&S->h, index, dim);
            float u1 = halton(&S->h, index, dim);
            sphere_cone(LM, seen, u0, u1, lp, ln, pdf);
            return;
        }
    }
    int lt = LM->first_tri + halton_int(&S->h, index, dim, LM->tri_count);
    float temp = sqrtf(halton(&S->h, index, dim));
    float su = 1 - temp;
    float sv = temp * halton(&S->h, index, dim);
    int a = S->idx[3 * lt], b = S->idx[3 * lt + 1], c = S->idx[3 * lt + 2];
    *lp = vadd(vadd(vs(ld3(S->pos + 3 * a), su), vs(ld3(S->pos + 3 * b), sv)), vs(ld3(S->pos + 3 * c), 1.f - su - sv));
    *ln = tri_normal(S, LM, lt, su, sv);
    V3 l2s = vsub(seen, *lp);
    float lcos = fabsf(vdot(*ln, vnorm(l2s)));
    *pdf = vdot(l2s, l2s) / (lcos * LM->area);
}

/* TriangleMesh::pdf (Core/TriangleMesh.h:213-232) of a ray from o reaching the light at p, n. */
static float light_pdf_at(const OMesh* LM, V3 o, V3 p, V3 n) {
    if (LM->shape == 1) {
        V3 dv = vsub(o, v3(LM->sphere[0], LM->sphere[1], LM->sphere[2]));
        float d2 = vdot(dv, dv), r2 = LM->sphere[3] * LM->sphere[3];
        if (d2 > r2) {
            float cos_max = sqrtf(fmaxf(0.f, 1.f - r2 / d2));
            return (float)(1.f / (2.f * M_PI * (1 - cos_max)));
        }
    }
    V3 l2s = vsub(o, p);
    float c = fabsf(vdot(n, vnorm(l2s)));
    return vdot(l2s, l2s) / (c * LM->area);
}

/* One camera sample through the integrator's bounce loop.  Returns the path's radiance. */
static V3 trace_path(const Scene* S, uint64_t index, V3 ro, V3 rd, int max_depth) {
    V3 res = v3(0, 0, 0), thr = v3(1, 1, 1);
    float mat_pdf = 1;
    int delta = 1;
    int dim0 = 0;
    for (int depth = 0; depth < max_depth; ++depth) {
        float o[3] = {ro.x, ro.y, ro.z}, d[3] = {rd.x, rd.y, rd.z};
        float t, u, v;
        int prim = orc_closest_one(S->nodes, S->pos, S->idx, o, d, &t, &u, &v);
        if (prim < 0) { /* intersectScene: the environment, without an MIS weight */
            if (S->env >= 0) res = vadd(res, vmul(env_eval(S, &S->lights[S->env], rd), thr));
            break;
        }
        const int mesh = S->tri_mesh[prim];
        const OMesh* M = &S->meshes[mesh];
        V3 pos = vadd(ro, vs(rd, t));
        V3 nrm = tri_normal(S, M, prim, u, v);
        if (M->light >= 0) { /* emission at the hit */
            const OLight* L = &S->lights[M->light];
            V3 Le = vdot(rd, nrm) >= 0 ? v3(0, 0, 0) : ld3(L->L);
            if (delta) {
                res = vadd(res, vmul(Le, thr));
            } else if (depth > 0) {
                float lpdf = light_pdf_at(&S->meshes[L->mesh], ro, pos, nrm);
                float w = mis_power(mat_pdf, lpdf);
                if (isfinite(w)) res = vadd(res, vs(vmul(Le, thr), w));
            }
        }
        const OMaterial* mat = &S->mats[M->material];
        Bsdf B = make_bsdf(mat);
        if (mat->kd_tex >= 0 && (mat->type == M_MATTE || mat->type == M_PLASTIC || mat->type == M_SUBSTRATE)) {
            float tu, tv;
            hit_texcoord(S, prim, u, v, &tu, &tv);
            V3 tx = tex_read(&S->textures[mat->kd_tex], tu, tv);
            B.kd = mat->type == M_MATTE ? vmul(B.kd, tx) : tx;
        }
        Frame fr = make_frame(nrm);
        V3 wo = to_local(&fr, vs(rd, -1.f));
        /* light sample: randInt(lights), rand4 (unused), then the light's own sample */
        int dim = dim0;
        int li = halton_int(&S->h, index, &dim, S->n_lights);
        dim += 4;
        const OLight* L = &S->lights[li];
        V3 dir, incident;
        float lpdf, limit;
        int target;
        if (L->kind == 1) { /* EnvironmentMap::sampleRayToPoint, uniformSampleSphere as written */
            float a0 = halton(&S->h, index, &dim), a1 = halton(&S->h, index, &dim);
            float a = (float)(a0 * 2 * M_PI), b = (float)((a1 - 0.5) * M_PI);
            dir = v3(cosf(b) * cosf(a), sinf(b), cosf(b) * sinf(a));
            lpdf = (float)(1.f / (4.f * M_PI));
            incident = env_eval(S, L, dir);
            limit = INFINITY;
            target = -1;
        } else {
            V3 lp, ln;
            light_sample(S, &S->meshes[L->mesh], pos, index, &dim, &lp, &ln, &lpdf);
            dir = vnorm(vsub(lp, pos));
            incident = vdot(dir, ln) >= 0 ? v3(0, 0, 0) : ld3(L->L);
            V3 dl = vsub(lp, pos);
            limit = sqrtf(vdot(dl, dl));
            target = L->mesh;
        }
        if (isfinite(lpdf)) {
            V3 wi = to_local(&fr, dir);
            float w = S->direct ? 1.f : mis_power(lpdf, bsdf_pdf(&B, wi, wo));
            float cosine = fabsf(vdot(dir, nrm));
            V3 mult = vdivs(vs(thr, (float)S->n_lights), lpdf);
            V3 contrib = vs(vmul(vs(vmul(incident, bsdf_eval(&B, wi, wo)), cosine), mult), w);
            if (!vzero(contrib)) {
                float so[3] = {pos.x, pos.y, pos.z}, sd[3] = {dir.x, dir.y, dir.z};
                if (orc_any_one(S->nodes, S->pos, S->idx, S->tri_mesh, so, sd, limit, mesh, target) == 0)
                    res = vadd(res, contrib);
            }
        }
        /* continuation */
        dim = dim0 + S->cont_dim;
        if (depth > 3) {
            float q = 1;
            q = fminf(q, 1 - thr.x);
            q = fminf(q, 1 - thr.y);
            q = fminf(q, 1 - thr.z);
            q = fmaxf(q, 0.05f);
            if (halton(&S->h, index, &dim) < q) break;
            thr = vdivs(thr, 1.f - q);
        }
        float u0 = halton(&S->h, index, &dim);
        float u1 = halton(&S->h, index, &dim);
        V3 wi;
        float p = 0;
        V3 f = bsdf_sample(&B, u0, u1, wo, &wi, &p);
        V3 nd = to_world(&fr, wi);
        if (vzero(f)) thr = v3(0, 0, 0);
        else thr = vdivs(vs(vmul(thr, f), fabsf(vdot(nd, nrm))), p);
        if (vzero(thr)) break;
        mat_pdf = p;
        delta = bsdf_delta(&B);
        ro = vadd(pos, vs(nd, 0.001f));
        rd = nd;
        dim0 += S->cont_dim + 2 + (depth > 3 ? 1 : 0);
    }
    return res;
}

/* TriangleMesh::computeArea: float sum of half cross-product lengths, in triangle order. */
static float mesh_area(const float* pos, const int32_t* idx, int first, int count) {
    float area = 0;
    for (int t = first; t < first + count; ++t) {
        V3 p0 = ld3(pos + 3 * idx[3 * t]), p1 = ld3(pos + 3 * idx[3 * t + 1]), p2 = ld3(pos + 3 * idx[3 * t + 2]);
        V3 c = vcross(vsub(p1, p0), vsub(p2, p0));
        area += sqrtf(c.x * c.x + c.y * c.y + c.z * c.z) * 0.5f;
    }
    return area;
}

/* Renders camera samples [first, first + count) of a W x H x spp image (pixel-major sample
 * numbering, as the reference's single sppBySpp round) and splats them into film_sum (3 per
 * pixel) / film_w (1 per pixel), which the caller zeroes.  meshes[].area is recomputed here.
 * Samples are traced in parallel (OpenMP) and splatted in sample order. */
int orc_render_path(const ONode* nodes, const float* pos, const int32_t* idx, const float* nrm,
                    const int32_t* tri_mesh, OMesh* meshes, int n_meshes, const OMaterial* mats,
                    const OLight* lights, int n_lights, const float* c2w, float fov_deg, int width, int height,
                    int spp, int max_depth, float xw, float yw, int64_t first, int64_t count, float* film_sum,
                    float* film_w, int direct, const float* uv, const OTexture* textures, int env) {
    if (n_lights <= 0 || width <= 0 || height <= 0 || spp <= 0) return -1;
    unsigned csr = _mm_getcsr();
    _mm_setcsr(csr | 0x8040); /* FTZ | DAZ, as the device build */
    Scene S;
    S.nodes = nodes;
    S.pos = pos;
    S.idx = idx;
    S.nrm = nrm;
    S.tri_mesh = tri_mesh;
    for (int m = 0; m < n_meshes; ++m) meshes[m].area = mesh_area(pos, idx, meshes[m].first_tri, meshes[m].tri_count);
    S.meshes = meshes;
    S.mats = mats;
    S.lights = lights;
    S.n_lights = n_lights;
    S.direct = direct;
    if (direct) max_depth = 1;
    S.uv = uv;
    S.textures = textures;
    S.env = env;
    S.cont_dim = 7;
    for (int l = 0; l < n_lights; ++l)
        if (lights[l].kind == 0) S.cont_dim = 8;
    int64_t plen = orc_halton_tables(S.h.primes, S.h.start, NULL);
    S.h.perms = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)plen);
    orc_halton_tables(S.h.primes, S.h.start, S.h.perms);
    float fov = fov_deg * 3.14159265358979323846f / 180.f;
    float depth = height <= width ? (height / 2.f) / tanf(fov / 2.f) : (width / 2.f) / tanf(fov / 2.f);
    const int64_t total = (int64_t)width * height * spp;
    if (first + count > total) count = total - first;
    float* res = (float*)malloc(sizeof(float) * 5 * (size_t)(count > 0 ? count : 1));
#pragma omp parallel
    {
        _mm_setcsr(_mm_getcsr() | 0x8040);
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < count; ++i) {
            int64_t s = first + i;
            int64_t pixel = s / spp;
            int x = (int)(pixel % width), y = (int)(pixel / width);
            uint64_t index = (uint64_t)pixel * (uint64_t)spp + (uint64_t)(s % spp);
            int dim = 0;
            float sx = x + halton(&S.h, index, &dim);
            float sy = y + halton(&S.h, index, &dim);
            V3 pl = v3(sx - width / 2.f, height / 2.f - sy, depth);
            V3 o = apply_pt(c2w, v3(0, 0, 0));
            V3 d = vnorm(vsub(apply_pt(c2w, pl), o));
            V3 r = trace_path(&S, index, o, d, max_depth);
            res[5 * i] = r.x;
            res[5 * i + 1] = r.y;
            res[5 * i + 2] = r.z;
            res[5 * i + 3] = sx;
            res[5 * i + 4] = sy;
        }
    }
    for (int64_t i = 0; i < count; ++i) {
        float r0 = res[5 * i], r1 = res[5 * i + 1], r2 = res[5 * i + 2], sx = res[5 * i + 3], sy = res[5 * i + 4];
        if (!isfinite(r0) || !isfinite(r1) || !isfinite(r2)) continue;
        int x0 = (int)floorf(sx - xw), x1 = (int)ceilf(sx + xw);
        int y0 = (int)floorf(sy - yw), y1 = (int)ceilf(sy + yw);
        for (int x = x0; x <= x1; ++x)
            for (int y = y0; y <= y1; ++y) {
                if (x >= width || y >= height || x < 0 || y < 0) continue;
                if (fabsf(x - sx) > xw || fabsf(y - sy) > yw) continue;
                int p = y * width + x;
                film_sum[3 * p] += r0;
                film_sum[3 * p + 1] += r1;
                film_sum[3 * p + 2] += r2;
                film_w[p] += 1.f;
            }
    }
    free(res);
    free(S.h.perms);
    _mm_setcsr(csr);
    return 0;
}

/* GGX::roughnessToAlpha (BSDFs/MicrofacetDistribution.h:57-63), host float arithmetic. */
float orc_roughness_to_alpha(float roughness) {
    roughness = fmaxf(roughness, 1e-3f);
    float x = logf(roughness);
    return 1.62142f + 0.819955f * x + 0.1734f * x * x + 0.0171201f * x * x * x + 0.000640711f * x * x * x * x;
}
