/*
 * bte_oracle.c -- ORACLE (test infrastructure only; the product never links,
 * imports or executes it).  CPU restatement of Blue Truth Engine's wavefront
 * path tracer: RNG, camera, the five BSDFs, emitter sampling, env-map
 * sampling, NEE/MIS, scatter, Russian roulette, accumulation and display
 * packing, each function following the reference file:line cited beside it
 * (paths relative to the reference project root), operation for operation so
 * that floating-point results agree bit-for-bit.
 *
 * The reference traces rays with OptiX (closed library, RT cores); the oracle
 * defines closest hit / occlusion with the watertight ray-triangle test of
 * Woop, Benthin and Wald (JCGT 2013), closest hit resolved by (t, triangle
 * index), in the interval [1e-4, tmax] used by rt_optix_shading.cuh:57-95.
 *
 * Shadow contributions are summed in the megakernel's order (emitter hit,
 * area NEE, spotlights in index order, env NEE: rt_optix_shading.cuh:412-447),
 * which the GPU reproduces deterministically instead of the reference's
 * racing float atomicAdd (src/wavefront/ray_connect.cu:67-69).
 *
 * Texture fetches (tex2D) are emulated with the CUDA Programming Guide's
 * documented linear-filtering formula (texel-centre offset of 0.5, weights in
 * 9-bit fixed point with 8 fractional bits).
 *
 * Deviation pinned on both sides: M_PI in rt_env_map.cuh:26-28 is taken as
 * the float literal (FP32 semantics); rsqrtf in normalize3 is 1.0f/sqrtf.
 *
 * Build: gcc -O2 -ffp-contract=off (see oracle/Makefile).
 */
#include "bte_oracle.h"
#include "bte_oracle_math.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef BTE_ORACLE_LIBM
#define O_SINF sinf
#define O_COSF cosf
#define O_TANF tanf
#define O_EXPF expf
#define O_LOGF logf
#define O_POWF powf
#define O_ATAN2F atan2f
#define O_ACOSF acosf
#define O_POW5(x) powf((x), 5)
#define O_POW2(x) powf((x), 2)
#else
#define O_SINF om_sinf
#define O_COSF om_cosf
#define O_TANF om_tanf
#define O_EXPF om_expf
#define O_LOGF om_logf
#define O_POWF om_powf
#define O_ATAN2F om_atan2f
#define O_ACOSF om_acosf
#define O_POW5(x) om_pow5f(x)
#define O_POW2(x) om_pow2f(x)
#endif

int or_math_mode(void)
{
#ifdef BTE_ORACLE_LIBM
    return 1;
#else
    return 0;
#endif
}

/* rt_constants.cuh:11-19 */
#define O_RT_EPSILON 1e-4f
/* rt_bsdf.cuh:11-12 */
#define O_PI 3.14159265358979323846f
#define O_INV_PI (1.0f / O_PI)
/* rt_env_map.cuh:26-28 (FP32 literal) */
#define O_MPI 3.14159265358979323846f
/* rt_bsdf_microfacet.cuh:11 */
#define O_AZIMUTH (1.0f / (2.0f * O_PI))

/* ------------------------------------------------------------------ */
/* vector helpers -- rt_cuda_math.cuh:8-124                           */
/* ------------------------------------------------------------------ */
static inline OF3 f3(float x, float y, float z) { OF3 r = {x, y, z}; return r; }
static inline OF3 sub3(OF3 a, OF3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline OF3 add3(OF3 a, OF3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline OF3 mul3s(OF3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
static inline OF3 mul3v(OF3 a, OF3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline OF3 div3(OF3 a, float s)
{
    if (s == 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float inv = 1.0f / s;
    return f3(a.x * inv, a.y * inv, a.z * inv);
}
static inline float dot3(OF3 a, OF3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline OF3 cross3(OF3 a, OF3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline OF3 normalize3(OF3 v)
{
    const float len2 = dot3(v, v);
    if (len2 <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float invLen = 1.0f / sqrtf(len2);
    return mul3s(v, invLen);
}
static inline float length3(OF3 v) { return sqrtf(fmaxf(0.0f, dot3(v, v))); }
static inline float distance3(OF3 a, OF3 b) { return length3(sub3(a, b)); }
static inline float maxCoeff3(OF3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }

typedef struct { OF3 t, b, n; } OFrame;
static inline OFrame makeFrame(OF3 normal)
{
    OFrame f;
    f.n = normalize3(normal);
    const OF3 a = (fabsf(f.n.z) < 0.999f) ? f3(0.0f, 0.0f, 1.0f) : f3(1.0f, 0.0f, 0.0f);
    f.t = normalize3(cross3(a, f.n));
    f.b = cross3(f.n, f.t);
    return f;
}
static inline OF3 toLocal(const OFrame* f, OF3 v) { return f3(dot3(v, f->t), dot3(v, f->b), dot3(v, f->n)); }
static inline OF3 toWorld(const OFrame* f, OF3 v)
{
    return add3(add3(mul3s(f->t, v.x), mul3s(f->b, v.y)), mul3s(f->n, v.z));
}
static inline OF3 toLocalN(OF3 n, OF3 v) { OFrame f = makeFrame(n); return toLocal(&f, v); }
static inline OF3 toWorldN(OF3 n, OF3 v) { OFrame f = makeFrame(n); return toWorld(&f, v); }

/* ------------------------------------------------------------------ */
/* RNG -- rt_rng.cuh:8-52                                             */
/* ------------------------------------------------------------------ */
uint32_t or_hash_uint(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static inline uint32_t rngMake(uint32_t seed) { return seed ? seed : 1u; }
static inline uint32_t rngNextU32(uint32_t* s)
{
    uint32_t x = *s;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    *s = x;
    return x;
}
static inline float rngNextFloat01(uint32_t* s)
{
    const uint32_t u = rngNextU32(s) >> 8;
    return (float)u * (1.0f / 16777216.0f);
}

void or_rng_stream(uint32_t seed, int n, uint32_t* outU32, float* outF)
{
    uint32_t s = rngMake(seed);
    uint32_t s2 = s;
    for (int i = 0; i < n; ++i) {
        if (outU32) outU32[i] = rngNextU32(&s);
        if (outF) outF[i] = rngNextFloat01(&s2);
    }
}

/* ------------------------------------------------------------------ */
/* texture emulation (tex2D, linear filtering, normalized coordinates) */
/* ------------------------------------------------------------------ */
/* Weight quantisation: 9-bit fixed point with 8 fractional bits. */
static inline float o_tex_weight(float frac)
{
    return floorf(frac * 256.0f + 0.5f) * (1.0f / 256.0f);
}
static inline int o_wrap(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
static inline int o_clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

/* Float4 texture, address mode x = wrap, y = wrap (wrapV=1) or clamp (0). */
static OF4 o_tex2d_f4(const float* texels, int w, int h, int wrapV, float u, float v)
{
    float x = u, y = v;
    x = x - floorf(x);                                   /* wrap */
    if (wrapV) y = y - floorf(y);
    else       y = fminf(fmaxf(y, 0.0f), 1.0f);          /* clamp */
    const float xb = x * (float)w - 0.5f;
    const float yb = y * (float)h - 0.5f;
    const float fx0 = floorf(xb), fy0 = floorf(yb);
    const float a = o_tex_weight(xb - fx0);
    const float b = o_tex_weight(yb - fy0);
    const int ix = (int)fx0, iy = (int)fy0;
    const int x0 = o_wrap(ix, w), x1 = o_wrap(ix + 1, w);
    const int y0 = wrapV ? o_wrap(iy, h) : o_clampi(iy, h);
    const int y1 = wrapV ? o_wrap(iy + 1, h) : o_clampi(iy + 1, h);
    const float* t00 = texels + ((size_t)y0 * w + x0) * 4;
    const float* t10 = texels + ((size_t)y0 * w + x1) * 4;
    const float* t01 = texels + ((size_t)y1 * w + x0) * 4;
    const float* t11 = texels + ((size_t)y1 * w + x1) * 4;
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    OF4 r;
    r.x = ((w00 * t00[0] + w10 * t10[0]) + w01 * t01[0]) + w11 * t11[0];
    r.y = ((w00 * t00[1] + w10 * t10[1]) + w01 * t01[1]) + w11 * t11[1];
    r.z = ((w00 * t00[2] + w10 * t10[2]) + w01 * t01[2]) + w11 * t11[2];
    r.w = ((w00 * t00[3] + w10 * t10[3]) + w01 * t01[3]) + w11 * t11[3];
    return r;
}

/* RGBA8 texture read as normalized float (value / 255), wrap/wrap. */
static OF4 o_tex2d_rgba8(const uint8_t* px, int w, int h, float u, float v)
{
    float x = u - floorf(u), y = v - floorf(v);
    const float xb = x * (float)w - 0.5f;
    const float yb = y * (float)h - 0.5f;
    const float fx0 = floorf(xb), fy0 = floorf(yb);
    const float a = o_tex_weight(xb - fx0);
    const float b = o_tex_weight(yb - fy0);
    const int ix = (int)fx0, iy = (int)fy0;
    const int x0 = o_wrap(ix, w), x1 = o_wrap(ix + 1, w);
    const int y0 = o_wrap(iy, h), y1 = o_wrap(iy + 1, h);
    const uint8_t* t00 = px + ((size_t)y0 * w + x0) * 4;
    const uint8_t* t10 = px + ((size_t)y0 * w + x1) * 4;
    const uint8_t* t01 = px + ((size_t)y1 * w + x0) * 4;
    const uint8_t* t11 = px + ((size_t)y1 * w + x1) * 4;
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    const float k = 1.0f / 255.0f;
    float c[4];
    for (int i = 0; i < 4; ++i) {
        c[i] = ((w00 * ((float)t00[i] * k) + w10 * ((float)t10[i] * k)) + w01 * ((float)t01[i] * k))
               + w11 * ((float)t11[i] * k);
    }
    OF4 r = {c[0], c[1], c[2], c[3]};
    return r;
}

void or_tex_sample_f4(const float* texels, int w, int h, int wrapV, float u, float v, float out[4])
{
    OF4 r = o_tex2d_f4(texels, w, h, wrapV, u, v);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

void or_tex_sample_rgba8(const uint8_t* px, int w, int h, float u, float v, float out[4])
{
    OF4 r = o_tex2d_rgba8(px, w, h, u, v);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

void or_tex_float4(const float* texels, int w, int h, int wrapV, const float* uv, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        OF4 r = o_tex2d_f4(texels, w, h, wrapV, uv[2 * i], uv[2 * i + 1]);
        out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
    }
}

/* ------------------------------------------------------------------ */
/* BSDFs -- rt_bsdf.cuh and rt_bsdf_*.cuh                             */
/* ------------------------------------------------------------------ */
typedef struct { OF3 wi, wo; int measure; float eta, rndExtra; } OBRec; /* rt_bsdf.cuh:19-25 */
#define O_ESOLID 1

/* rt_bsdf_diffuse.cuh:15-24 */
static inline OF3 o_sqCosHemi(float u1, float u2)
{
    const float r = sqrtf(fmaxf(u1, 0.0f));
    const float phi = 2.0f * O_PI * u2;
    const float x = r * O_COSF(phi);
    const float y = r * O_SINF(phi);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    return f3(x, y, z);
}
/* rt_bsdf_diffuse.cuh:27-62 */
static OF3 o_evalDiffuse(const OBsdf* b, const OBRec* r)
{
    if (r->measure != O_ESOLID || r->wi.z <= 0.0f || r->wo.z <= 0.0f) return f3(0, 0, 0);
    return mul3s(f3(b->p0.x, b->p0.y, b->p0.z), O_INV_PI);
}
static float o_pdfDiffuse(const OBRec* r)
{
    if (r->measure != O_ESOLID || r->wi.z <= 0.0f || r->wo.z <= 0.0f) return 0.0f;
    return O_INV_PI * r->wo.z;
}
static OF3 o_sampleDiffuse(const OBsdf* b, OBRec* r, float u1, float u2)
{
    if (r->wi.z <= 0.0f) return f3(0, 0, 0);
    r->measure = O_ESOLID;
    r->wo = o_sqCosHemi(u1, u2);
    r->eta = 1.0f;
    return f3(b->p0.x, b->p0.y, b->p0.z);
}

/* rt_bsdf_mirror.cuh:13-33 */
static OF3 o_sampleMirror(const OBsdf* b, OBRec* r)
{
    r->wo = f3(-r->wi.x, -r->wi.y, r->wi.z);
    r->eta = 1.0f;
    r->measure = O_ESOLID;
    return f3(b->p0.x, b->p0.y, b->p0.z);
}

/* rt_bsdf_dielectric.cuh:13-31 */
static float o_fresnelDielectric(float cosThetaI, float etaI, float etaT)
{
    if (cosThetaI < 0.0f) {
        float tmp = etaI; etaI = etaT; etaT = tmp;
        cosThetaI = -cosThetaI;
    }
    float sinThetaT = (etaI / etaT) * sqrtf(fmaxf(0.0f, 1.0f - cosThetaI * cosThetaI));
    if (sinThetaT >= 1.0f) return 1.0f;
    float cosThetaT = sqrtf(fmaxf(0.0f, 1.0f - sinThetaT * sinThetaT));
    float Rs = (etaI * cosThetaI - etaT * cosThetaT) / (etaI * cosThetaI + etaT * cosThetaT);
    float Rp = (etaT * cosThetaI - etaI * cosThetaT) / (etaT * cosThetaI + etaI * cosThetaT);
    return (Rs * Rs + Rp * Rp) * 0.5f;
}
/* rt_bsdf_dielectric.cuh:51-103 */
static OF3 o_sampleDielectric(const OBsdf* b, OBRec* r, float u1)
{
    r->measure = O_ESOLID;
    OF3 res = f3(1.0f, 1.0f, 1.0f);
    float cosThetaI = r->wi.z;
    const float fr = o_fresnelDielectric(cosThetaI, b->p1.y, b->p1.x);
    if (u1 < fr) {
        r->wo = f3(-r->wi.x, -r->wi.y, r->wi.z);
        r->eta = 1.0f;
    } else {
        float ratio;
        OF3 nrm = f3(0.0f, 0.0f, 1.0f);
        if (cosThetaI > 0) {
            ratio = b->p1.y / b->p1.x;
        } else {
            ratio = b->p1.x / b->p1.y;
            nrm = f3(0.0f, 0.0f, -1.0f);
        }
        cosThetaI = fabsf(cosThetaI);
        float rootTerm = 1.0f - (ratio * ratio) * (1.0f - cosThetaI * cosThetaI);
        float dia = ratio * cosThetaI - sqrtf(rootTerm);
        r->wo = f3(-ratio * r->wi.x + dia * nrm.x, -ratio * r->wi.y + dia * nrm.y,
                   -ratio * r->wi.z + dia * nrm.z);
        r->eta = 1.0f / ratio;
        float w = ratio * ratio;
        res = f3(w, w, w);
    }
    return res;
}

/* rt_bsdf_microfacet.cuh:23-185 */
static inline float o_tanThetaMf(OF3 w)
{
    const float ct = w.z;
    const float sin2 = fmaxf(0.0f, 1.0f - ct * ct);
    const float cos2 = ct * ct;
    if (cos2 <= 0.0f) return 0.0f;
    return sqrtf(sin2 / cos2);
}
static inline OF3 o_sqBeckmann(float u1, float u2, float alpha)
{
    const float phi = 2.0f * O_PI * u2;
    const float tan2 = -alpha * alpha * O_LOGF(fmaxf(1.0e-6f, 1.0f - u1));
    const float cosT = 1.0f / sqrtf(1.0f + tan2);
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    return f3(sinT * O_COSF(phi), sinT * O_SINF(phi), cosT);
}
static inline float o_sqBeckmannPdf(OF3 m, float alpha)
{
    if (m.z <= 0.0f) return 0.0f;
    const float tanT = o_tanThetaMf(m);
    const float a2 = alpha * alpha;
    const float c = m.z;
    const float c3 = c * c * c;
    return O_AZIMUTH * (2.0f * O_EXPF(-1.0f * tanT * tanT / a2)) / (a2 * c3);
}
static inline float o_shadowMask(const OBsdf* b, OF3 wv, OF3 wh)
{
    const float c = dot3(wv, wh) / wv.z;
    if (c <= 0.0f) return 0.0f;
    const float bb = 1.0f / (b->p1.x * o_tanThetaMf(wv));
    if (bb < 1.6f) return ((3.535f * bb) + 2.181f * bb * bb) / (1.0f + (2.276f * bb) + 2.577f * bb * bb);
    return 1.0f;
}
static OF3 o_evalMicrofacet(const OBsdf* b, const OBRec* r)
{
    if (r->measure != O_ESOLID || r->wi.z <= 0.0f || r->wo.z <= 0.0f) return f3(0, 0, 0);
    const float alpha = b->p1.x;
    const OF3 diffuse = f3(b->p0.x * O_INV_PI, b->p0.y * O_INV_PI, b->p0.z * O_INV_PI);
    const OF3 wh = normalize3(add3(r->wi, r->wo));
    const float tanH = o_tanThetaMf(wh);
    const float cosH = wh.z;
    const float num = 2.0f * O_EXPF(-1.0f * tanH * tanH / (alpha * alpha));
    const float den = alpha * alpha * cosH * cosH * cosH;
    const float D = O_AZIMUTH * num / den;
    const float F = o_fresnelDielectric(dot3(wh, r->wi), b->p1.z, b->p1.y);
    const float G = o_shadowMask(b, r->wi, wh) * o_shadowMask(b, r->wo, wh);
    const float ci = r->wi.z, co = r->wo.z;
    const float ecf = 4.0f * ci * cosH * co;
    const float spec = b->p1.w * (D * F * G) / ecf;
    return f3(diffuse.x + spec, diffuse.y + spec, diffuse.z + spec);
}
static float o_pdfMicrofacet(const OBsdf* b, const OBRec* r)
{
    if (r->measure != O_ESOLID || r->wi.z <= 0.0f || r->wo.z <= 0.0f) return 0.0f;
    const float cosPdf = (r->wo.z <= 0.0f) ? 0.0f : O_INV_PI * r->wo.z;
    const OF3 wh = normalize3(add3(r->wi, r->wo));
    const float bp = o_sqBeckmannPdf(wh, b->p1.x);
    const float jac = 1.0f / (4.0f * dot3(wh, r->wo));
    return b->p1.w * bp * jac + (1.0f - b->p1.w) * cosPdf;
}
static OF3 o_sampleMicrofacet(const OBsdf* b, OBRec* r, float u1, float u2)
{
    if (r->wi.z <= 0.0f) return f3(0, 0, 0);
    float sx = u1;
    int refl;
    if (sx < b->p1.w) { refl = 0; sx = sx / b->p1.w; }
    else { refl = 1; sx = (sx - b->p1.w) / (1.0f - b->p1.w); }
    r->measure = O_ESOLID;
    r->eta = 1.0f;
    if (refl == 0) {
        const OF3 m = o_sqBeckmann(sx, u2, b->p1.x);
        r->wo = sub3(mul3s(m, 2.0f * dot3(r->wi, m)), r->wi);
    } else {
        r->wo = o_sqCosHemi(sx, u2);
    }
    if (r->wo.z <= 0.0f) return f3(0, 0, 0);
    const float p = o_pdfMicrofacet(b, r);
    if (p <= 0.0f) return f3(0, 0, 0);
    return mul3s(o_evalMicrofacet(b, r), r->wo.z / p);
}

/* ---- Disney: rt_bsdf_disney.cuh:16-892 ---- */
#define DBASE(b) f3((b)->p0.x, (b)->p0.y, (b)->p0.z)
#define DROUGH(b) ((b)->p0.w)
#define DMETAL(b) ((b)->p1.x)
#define DSPEC(b) ((b)->p1.y)
#define DSPECTRANS(b) ((b)->p1.z)
#define DSPECTINT(b) ((b)->p1.w)
#define DSHEEN(b) ((b)->p2.x)
#define DSHEENTINT(b) ((b)->p2.y)
#define DSUBSURF(b) ((b)->p2.z)
#define DANISO(b) ((b)->p2.w)
#define DCLEAR(b) ((b)->p3.x)
#define DCLEARGLOSS(b) ((b)->p3.y)
#define DETA(b) ((b)->p3.z)

static inline OF3 o_dsqrt3(OF3 c) { return f3(sqrtf(fmaxf(0.0f, c.x)), sqrtf(fmaxf(0.0f, c.y)), sqrtf(fmaxf(0.0f, c.z))); }

/* :42-56 */
static inline float o_diffF90(const OBsdf* b, float h) { return 0.5f + (2.0f * DROUGH(b) * h * h); }
static inline float o_diffF(float c, float f90) { return 1.0f + ((f90 - 1.0f) * O_POW5(1.0f - c)); }
static inline float o_ssF90(const OBsdf* b, float h) { return DROUGH(b) * h * h; }
static inline float o_ssF(float c, float f90) { return 1.0f + ((f90 - 1.0f) * O_POW5(1.0f - c)); }

/* :59-104 */
static OF3 o_evalDiffuseLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z, co = r->wo.z;
    if (ci <= 0.0f || co <= 0.0f) return f3(0, 0, 0);
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float hDotWo = fabsf(dot3(wh, r->wo));
    float dfN = o_diffF90(b, hDotWo);
    float ssN = o_ssF90(b, hDotWo);
    OF3 cop = div3(DBASE(b), O_PI);
    OF3 base = mul3s(cop, o_diffF(ci, dfN) * o_diffF(co, dfN) * co);
    float ssDenom = fmaxf(1e-2f, ci + co);
    OF3 ss = mul3s(cop, 1.25f * (o_ssF(ci, ssN) * o_ssF(co, ssN) * ((1.0f / ssDenom) - 0.5f) + 0.5f) * co);
    return add3(mul3s(base, 1.0f - DSUBSURF(b)), mul3s(ss, DSUBSURF(b)));
}
/* :107-124 */
static float o_pdfDiffuseLobe(const OBRec* r)
{
    if (r->measure != O_ESOLID || r->wi.z <= 0 || r->wo.z <= 0) return 0.0f;
    return O_INV_PI * r->wo.z;
}
/* :127-146 */
static OF3 o_sampleDiffuseLobe(const OBsdf* b, OBRec* r, float u1, float u2)
{
    if (r->wi.z <= 0) return f3(0, 0, 0);
    r->measure = O_ESOLID;
    r->wo = o_sqCosHemi(u1, u2);
    r->eta = 1.0f;
    return div3(o_evalDiffuseLobe(b, r), o_pdfDiffuseLobe(r));
}

/* :150-184 */
static inline float o_schlickFresnel(float eta)
{
    float n = eta - 1.0f, d = eta + 1.0f;
    return (n * n) / (d * d);
}
static OF3 o_fresnelMetal(const OBsdf* b, float hDotWo)
{
    OF3 bc = DBASE(b);
    float lumi = 0.3f * bc.x + 0.6f * bc.y + 0.1f * bc.z;
    OF3 tint = f3(1.0f, 1.0f, 1.0f);
    if (lumi > 0) tint = div3(bc, lumi);
    float st = DSPECTINT(b);
    OF3 spec = f3((1.0f - st) + (st * tint.x), (1.0f - st) + (st * tint.y), (1.0f - st) + (st * tint.z));
    float coef = DSPEC(b) * o_schlickFresnel(DETA(b)) * (1.0f - DMETAL(b));
    OF3 clr = f3((coef * spec.x) + (bc.x * DMETAL(b)), (coef * spec.y) + (bc.y * DMETAL(b)),
                 (coef * spec.z) + (bc.z * DMETAL(b)));
    float sch = O_POW5(1.0f - hDotWo);
    return f3(clr.x + ((1.0f - clr.x) * sch), clr.y + ((1.0f - clr.y) * sch), clr.z + ((1.0f - clr.z) * sch));
}
/* :186-210 */
static inline float o_ggxD(OF3 wh, float ax, float ay)
{
    float den = O_PI * ax * ay *
                O_POW2(((wh.x * wh.x) / (ax * ax)) + ((wh.y * wh.y) / (ay * ay)) + (wh.z * wh.z));
    return 1.0f / den;
}
static inline float o_lambda(OF3 w, float ax, float ay)
{
    float axw = w.x * ax, ayw = w.y * ay;
    float num = sqrtf(1 + (((axw * axw) + (ayw * ayw)) / fmaxf(1e-8f, (w.z * w.z)))) - 1.0f;
    float lam = num / 2.0f;
    return 1.0f / (1.0f + lam);
}
static inline float o_smithG(OF3 wi, OF3 wo, float ax, float ay) { return o_lambda(wi, ax, ay) * o_lambda(wo, ax, ay); }

static inline void o_alpha(const OBsdf* b, float* ax, float* ay)
{
    float aspect = sqrtf(1.0f - (0.9f * DANISO(b)));
    *ax = fmaxf((float)0.0001, (DROUGH(b) * DROUGH(b)) / aspect);
    *ay = fmaxf((float)0.0001, (DROUGH(b) * DROUGH(b)) * aspect);
}

/* :213-241 */
static OF3 o_evalMetalLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z;
    if (ci <= 0.0f || r->wo.z <= 0.0f) return f3(0, 0, 0);
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float hDotWo = fabsf(dot3(wh, r->wo));
    float ax, ay; o_alpha(b, &ax, &ay);
    OF3 fm = o_fresnelMetal(b, hDotWo);
    float dm = o_ggxD(wh, ax, ay);
    float gm = o_smithG(r->wi, r->wo, ax, ay);
    return div3(mul3s(fm, dm * gm), (4 * ci));
}
/* :244-271 */
static float o_pdfMetalLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z;
    if (ci <= 0.0f || r->wo.z <= 0.0f) return 0.0f;
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float ax, ay; o_alpha(b, &ax, &ay);
    float dm = o_ggxD(wh, ax, ay);
    float gm = o_lambda(r->wi, ax, ay);
    float hDotWi = fabsf(dot3(wh, r->wi));
    float hDotWo = fabsf(dot3(wh, r->wo));
    return (dm * gm * hDotWi) / (ci * 4.0f * hDotWo);
}
/* Heitz visible-normal sampling block shared by :293-317 and :610-634 */
static OF3 o_vndf(OF3 w, float ax, float ay, float u1, float u2)
{
    OF3 vh = normalize3(f3(ax * w.x, ay * w.y, w.z));
    float pl = (vh.x * vh.x) + (vh.y * vh.y);
    OF3 o1 = f3(1.0f, 0.0f, 0.0f);
    if (pl > 0.0f) o1 = div3(f3(-1.0f * vh.y, vh.x, 0.0f), sqrtf(pl));
    OF3 o2 = cross3(vh, o1);
    float radius = sqrtf(u1);
    float phi = 2.0f * O_PI * u2;
    float t1 = radius * O_COSF(phi);
    float t2 = radius * O_SINF(phi);
    float skew = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - skew) * sqrtf(1.0f - (t1 * t1)) + (skew * t2);
    OF3 ph = add3(add3(mul3s(o1, t1), mul3s(o2, t2)), mul3s(vh, sqrtf(fmaxf(0.0f, 1 - (t1 * t1) - (t2 * t2)))));
    return normalize3(f3(ax * ph.x, ay * ph.y, fmaxf(0.0f, ph.z)));
}
/* :274-335 */
static OF3 o_sampleMetalLobe(const OBsdf* b, OBRec* r, float u1, float u2)
{
    if (r->wi.z <= 0.0f) return f3(0, 0, 0);
    r->measure = O_ESOLID;
    r->eta = 1.0f;
    float ax, ay; o_alpha(b, &ax, &ay);
    OF3 h = o_vndf(r->wi, ax, ay, u1, u2);
    r->wo = sub3(mul3s(h, 2.0f * dot3(r->wi, h)), r->wi);
    if (r->wo.z <= 0.0f) return f3(0, 0, 0);
    float hDotWo = fabsf(dot3(h, r->wo));
    OF3 fm = o_fresnelMetal(b, hDotWo);
    float gm = o_lambda(r->wo, ax, ay);
    return mul3s(fm, gm);
}
/* :339-363 */
static inline float o_fresnelClear(float hDotWo)
{
    float rr = (float)0.04;
    return rr + ((1.0f - rr) * O_POW5(1.0f - hDotWo));
}
static inline float o_clearD(const OBsdf* b, OF3 wh)
{
    float ir = ((1.0f - DCLEARGLOSS(b)) * 0.1f) + (DCLEARGLOSS(b) * 0.001f);
    float ir2 = ir * ir;
    float num = ir2 - 1.0f;
    float den = O_PI * O_LOGF(ir2) * (1.0f + ((ir2 - 1.0f) * (wh.z * wh.z)));
    return num / den;
}
/* :370-394 */
static OF3 o_evalClearLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z;
    if (ci <= 0.0f || r->wo.z <= 0.0f) return f3(0, 0, 0);
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float hDotWo = fabsf(dot3(wh, r->wo));
    float fc = o_fresnelClear(hDotWo);
    float dc = o_clearD(b, wh);
    float gc = o_lambda(r->wi, 0.25f, 0.25f) * o_lambda(r->wo, 0.25f, 0.25f);
    float den = 4.0f * ci;
    float cc = (fc * dc * gc) / den;
    return f3(cc, cc, cc);
}
/* :397-414 */
static float o_pdfClearLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z;
    if (ci <= 0.0f || r->wo.z <= 0.0f) return 0.0f;
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float dc = o_clearD(b, wh);
    float hDotWo = fabsf(dot3(wh, r->wo));
    return (dc * wh.z) / (4.0f * hDotWo);
}
/* :417-450 */
static OF3 o_sampleClearLobe(const OBsdf* b, OBRec* r, float u1, float u2)
{
    if (r->wi.z <= 0.0f) return f3(0, 0, 0);
    r->measure = O_ESOLID;
    float ir = ((1.0f - DCLEARGLOSS(b)) * 0.1f) + (DCLEARGLOSS(b) * 0.001f);
    float ir2 = ir * ir;
    float az = 2.0f * O_PI * u1;
    float ce2 = (1.0f - O_POWF(ir2, 1.0f - u2)) / (1.0f - ir2);
    float se = sqrtf(1.0f - ce2);
    float hz = sqrtf(ce2);
    float hy = se * O_SINF(az);
    float hx = se * O_COSF(az);
    OF3 wh = normalize3(f3(hx, hy, hz));
    r->wo = sub3(mul3s(wh, 2.0f * dot3(r->wi, wh)), r->wi);
    r->eta = 1.0f;
    if (r->wo.z <= 0.0f) return f3(0, 0, 0);
    return div3(o_evalClearLobe(b, r), o_pdfClearLobe(b, r));
}
/* :455-472 */
static inline float o_fresnelGlass(float hi, float ho, float ehi, float eho)
{
    hi = fabsf(hi); ho = fabsf(ho); ehi = fabsf(ehi); eho = fabsf(eho);
    float rsN = hi - eho, rsD = hi + eho;
    float rpN = ehi - ho, rpD = ehi + ho;
    float rs = rsN / rsD, rp = rpN / rpD;
    return 0.5f * ((rs * rs) + (rp * rp));
}
/* half vector of the glass lobe, :486-498 / :546-558 */
static inline OF3 o_glassHalf(const OBRec* r, float eta, float inNout)
{
    OF3 wh;
    if (inNout > 0.0f) wh = normalize3(add3(r->wi, r->wo));
    else wh = mul3s(normalize3(add3(r->wi, mul3s(r->wo, eta))), -1.0f);
    if (wh.z < 0.0f) wh = mul3s(wh, -1.0f);
    return wh;
}
/* :475-532 */
static OF3 o_evalGlassLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z, co = r->wo.z;
    float eta = DETA(b);
    if (ci < 0.0f) eta = 1.0f / eta;
    float inNout = ci * co;
    OF3 wh = o_glassHalf(r, eta, inNout);
    float hDotWi = dot3(wh, r->wi), hDotWo = dot3(wh, r->wo);
    float ehi = eta * hDotWi, eho = eta * hDotWo;
    float fg = o_fresnelGlass(hDotWi, hDotWo, ehi, eho);
    float ax, ay; o_alpha(b, &ax, &ay);
    float dg = o_ggxD(wh, ax, ay);
    float gg = o_smithG(r->wi, r->wo, ax, ay);
    if (inNout > 0.0f) {
        OF3 num = mul3s(DBASE(b), fg * dg * gg);
        float den = 4.0f * fabsf(ci);
        return div3(num, den);
    } else {
        OF3 num = mul3s(o_dsqrt3(DBASE(b)), (1.0f - fg) * dg * gg * fabsf(hDotWi * hDotWo));
        float den = fabsf(ci) * fmaxf(O_POW2(hDotWi + eho), 1e-4f);
        return div3(num, den);
    }
}
/* :535-588 */
static float o_pdfGlassLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z, co = r->wo.z;
    float eta = DETA(b);
    if (ci < 0.0f) eta = 1.0f / eta;
    float inNout = ci * co;
    OF3 wh = o_glassHalf(r, eta, inNout);
    float hDotWi = dot3(wh, r->wi), hDotWo = dot3(wh, r->wo);
    float fg = o_fresnelGlass(hDotWi, hDotWo, eta * hDotWi, eta * hDotWo);
    float ax, ay; o_alpha(b, &ax, &ay);
    float dg = o_ggxD(wh, ax, ay);
    float gg = o_lambda(r->wi, ax, ay);
    float common = (dg * gg * fabsf(hDotWi)) / fabsf(ci);
    if (inNout > 0.0f) return (common * fg) / (4.0f * fabsf(hDotWo));
    float jac = (eta * eta * fabsf(hDotWo)) / fmaxf(O_POW2(hDotWi + (eta * hDotWo)), 1e-4f);
    return (1.0f - fg) * common * jac;
}
/* :591-674 */
static OF3 o_sampleGlassLobe(const OBsdf* b, OBRec* r, float u1, float u2)
{
    float ci = r->wi.z;
    r->measure = O_ESOLID;
    float ax, ay; o_alpha(b, &ax, &ay);
    float eta = DETA(b);
    if (ci < 0.0f) eta = 1.0f / eta;
    OF3 wiU = (ci < 0.0f) ? mul3s(r->wi, -1.0f) : r->wi;
    OF3 h = o_vndf(wiU, ax, ay, u1, u2);
    if (ci < 0.0f) h = mul3s(h, -1.0f);
    float hDotWi = dot3(h, r->wi);
    float sin2T = (1.0f - hDotWi * hDotWi) / (eta * eta);
    float hDotWt = sqrtf(fmaxf(0.0f, 1.0f - sin2T));
    float fg = o_fresnelGlass(hDotWi, hDotWt, eta * hDotWi, eta * hDotWt);
    if (r->rndExtra < fg || sin2T >= 1.0f) {
        r->wo = sub3(mul3s(h, 2.0f * dot3(r->wi, h)), r->wi);
        r->eta = 1.0f;
    } else {
        r->wo = sub3(mul3s(h, (hDotWi / eta) - hDotWt), div3(r->wi, eta));
        r->wo = normalize3(r->wo);
        r->eta = eta;
    }
    float pdf = o_pdfGlassLobe(b, r);
    if (pdf == 0.0f) return f3(0, 0, 0);
    return div3(o_evalGlassLobe(b, r), pdf);
}
/* :679-709 */
static OF3 o_evalSheenLobe(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z, co = r->wo.z;
    if (ci <= 0.0f || co <= 0.0f) return f3(0, 0, 0);
    OF3 wh = normalize3(add3(r->wi, r->wo));
    float hDotWo = fabsf(dot3(wh, r->wo));
    OF3 bc = DBASE(b);
    float lumi = 0.3f * bc.x + 0.6f * bc.y + 0.1f * bc.z;
    OF3 tint = f3(1.0f, 1.0f, 1.0f);
    if (lumi > 0) tint = div3(bc, lumi);
    float st = DSHEENTINT(b);
    OF3 sh = f3((1.0f - st) + (st * tint.x), (1.0f - st) + (st * tint.y), (1.0f - st) + (st * tint.z));
    return mul3s(sh, O_POW5(1.0f - hDotWo) * co);
}
/* :758-787 */
static OF3 o_evalDisney(const OBsdf* b, const OBRec* r)
{
    float ci = r->wi.z;
    if (ci <= 0.0f) {
        if (DSPECTRANS(b) <= 0.0f) return f3(0, 0, 0);
        return o_evalGlassLobe(b, r);
    }
    float minMetal = (1.0f - DMETAL(b));
    float minST = (1.0f - DSPECTRANS(b));
    OF3 fd = mul3s(o_evalDiffuseLobe(b, r), minMetal * minST);
    OF3 fs = mul3s(o_evalSheenLobe(b, r), minMetal * DSHEEN(b));
    OF3 fm = mul3s(o_evalMetalLobe(b, r), (1.0f - (DSPECTRANS(b) * minMetal)));
    OF3 fc = mul3s(o_evalClearLobe(b, r), 0.25f * DCLEAR(b));
    OF3 fg = mul3s(o_evalGlassLobe(b, r), minMetal * DSPECTRANS(b));
    return add3(add3(add3(add3(fd, fm), fg), fc), fs);
}
/* :790-820 */
static float o_pdfDisney(const OBsdf* b, const OBRec* r)
{
    float minMetal = (1.0f - DMETAL(b));
    float minST = (1.0f - DSPECTRANS(b));
    float dW = minMetal * minST;
    float mW = 1.0f - (DSPECTRANS(b) * minMetal);
    float gW = minMetal * DSPECTRANS(b);
    float cW = 0.25f * DCLEAR(b);
    float wSum = dW + gW + mW + cW;
    float ci = r->wi.z;
    if (ci <= 0) {
        if (DSPECTRANS(b) <= 0.0f) return 0.0f;
        return o_pdfGlassLobe(b, r);
    }
    float pD = o_pdfDiffuseLobe(r);
    float pM = o_pdfMetalLobe(b, r);
    float pG = o_pdfGlassLobe(b, r);
    float pC = o_pdfClearLobe(b, r);
    return (dW * pD + gW * pG + mW * pM + cW * pC) / wSum;
}
/* :823-892 */
static OF3 o_sampleDisney(const OBsdf* b, OBRec* r, float u1, float u2)
{
    float ci = r->wi.z;
    if (ci <= 0.0f) {
        if (DSPECTRANS(b) <= 0.0f) return f3(0, 0, 0);
        o_sampleGlassLobe(b, r, u1, u2);
    } else {
        float minMetal = (1.0f - DMETAL(b));
        float dW = minMetal * (1.0f - DSPECTRANS(b));
        float sW = minMetal * DSPECTRANS(b);
        float mW = 1.0f - (DSPECTRANS(b) * minMetal);
        float cW = 0.25f * DCLEAR(b);
        float wSum = dW + sW + mW + cW;
        float rc = r->rndExtra;
        float dF = dW / wSum, sF = sW / wSum, mF = mW / wSum;
        if (rc < dF) {
            o_sampleDiffuseLobe(b, r, u1, u2);
        } else if (rc < dF + sF) {
            r->rndExtra = (sF > 0.0f) ? (rc - dF) / sF : 0.0f;
            o_sampleGlassLobe(b, r, u1, u2);
        } else if (rc < dF + sF + mF) {
            o_sampleMetalLobe(b, r, u1, u2);
        } else {
            o_sampleClearLobe(b, r, u1, u2);
        }
    }
    float pdf = o_pdfDisney(b, r);
    if (pdf < 1e-7f) return f3(0, 0, 0);
    return div3(o_evalDisney(b, r), pdf);
}

/* dispatchers -- rt_bsdf.cuh:42-84 */
static OF3 o_bsdfEval(const OBsdf* b, const OBRec* r)
{
    switch (b->type) {
    case O_BSDF_DIFFUSE: return o_evalDiffuse(b, r);
    case O_BSDF_MICROFACET: return o_evalMicrofacet(b, r);
    case O_BSDF_DISNEY: return o_evalDisney(b, r);
    default: return f3(0, 0, 0);   /* dielectric, mirror (delta), unknown */
    }
}
static float o_bsdfPdf(const OBsdf* b, const OBRec* r)
{
    switch (b->type) {
    case O_BSDF_DIFFUSE: return o_pdfDiffuse(r);
    case O_BSDF_MICROFACET: return o_pdfMicrofacet(b, r);
    case O_BSDF_DISNEY: return o_pdfDisney(b, r);
    default: return 0.0f;
    }
}
static OF3 o_bsdfSample(const OBsdf* b, OBRec* r, float u1, float u2)
{
    switch (b->type) {
    case O_BSDF_DIFFUSE: return o_sampleDiffuse(b, r, u1, u2);
    case O_BSDF_DIELECTRIC: return o_sampleDielectric(b, r, u1);
    case O_BSDF_MIRROR: return o_sampleMirror(b, r);
    case O_BSDF_MICROFACET: return o_sampleMicrofacet(b, r, u1, u2);
    case O_BSDF_DISNEY: return o_sampleDisney(b, r, u1, u2);
    default: return f3(0, 0, 0);
    }
}
static inline int o_isDiffuseClass(const OBsdf* b)
{
    return b->type == O_BSDF_DIFFUSE || b->type == O_BSDF_MICROFACET || b->type == O_BSDF_DISNEY;
}

void or_bsdf_eval(const OBsdf* b, const float* wi, const float* wo, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        OBRec r; memset(&r, 0, sizeof r);
        r.wi = f3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        r.wo = f3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        r.measure = O_ESOLID;
        OF3 v = o_bsdfEval(b, &r);
        out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
    }
}
void or_bsdf_pdf(const OBsdf* b, const float* wi, const float* wo, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        OBRec r; memset(&r, 0, sizeof r);
        r.wi = f3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        r.wo = f3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        r.measure = O_ESOLID;
        out[i] = o_bsdfPdf(b, &r);
    }
}
void or_bsdf_sample(const OBsdf* b, const float* wi, const float* u, float* outWo, float* outWeight,
                    float* outPdf, float* outEta, int n)
{
    for (int i = 0; i < n; ++i) {
        OBRec r; memset(&r, 0, sizeof r);
        r.wi = f3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        r.rndExtra = u[3 * i];
        OF3 w = o_bsdfSample(b, &r, u[3 * i + 1], u[3 * i + 2]);
        outWo[3 * i] = r.wo.x; outWo[3 * i + 1] = r.wo.y; outWo[3 * i + 2] = r.wo.z;
        outWeight[3 * i] = w.x; outWeight[3 * i + 1] = w.y; outWeight[3 * i + 2] = w.z;
        outPdf[i] = o_bsdfPdf(b, &r);
        outEta[i] = r.eta;
    }
}

/* ------------------------------------------------------------------ */
/* material fetch -- rt_material.cuh:15-59                            */
/* ------------------------------------------------------------------ */
static OBsdf o_loadBsdf(const OScene* s, int tri, OF2 uv)
{
    OBsdf b = s->bsdfs[s->triBsdfIds[tri]];
    if (s->texPixels != NULL && s->triMaterialIds != NULL) {
        const int m = s->triMaterialIds[tri];
        if (m >= 0 && m < s->textureCount) {
            if (s->texPixels[m] != NULL) {
                OF4 t = o_tex2d_rgba8(s->texPixels[m], s->texW[m], s->texH[m], uv.x, uv.y);
                b.p0.x = t.x; b.p0.y = t.y; b.p0.z = t.z;
                if (b.type == O_BSDF_MICROFACET) b.p1.w = 1.0f - fmaxf(b.p0.x, fmaxf(b.p0.y, b.p0.z));
            }
            if (s->mrPixels != NULL) {
                if (s->mrPixels[m] != NULL && b.type == O_BSDF_DISNEY) {
                    OF4 mr = o_tex2d_rgba8(s->mrPixels[m], s->mrW[m], s->mrH[m], uv.x, uv.y);
                    b.p0.w *= mr.y;
                    b.p1.x *= mr.z;
                }
            }
        }
    }
    return b;
}

/* ------------------------------------------------------------------ */
/* environment map -- rt_env_map.cuh:36-199                           */
/* ------------------------------------------------------------------ */
static inline OF2 o_dirToEquirect(OF3 d, float rot)
{
    float phi = O_ATAN2F(d.z, d.x) + rot;
    float theta = O_ACOSF(fminf(fmaxf(d.y, -1.0f), 1.0f));
    phi = fmodf(phi + O_MPI, 2.0f * O_MPI);
    if (phi < 0.0f) phi += 2.0f * O_MPI;
    phi -= O_MPI;
    OF2 r = {(phi + O_MPI) / (2.0f * O_MPI), theta / O_MPI};
    return r;
}
static inline OF3 o_equirectToDir(float u, float v, float rot)
{
    float phi = u * 2.0f * O_MPI - O_MPI - rot;
    float theta = v * O_MPI;
    float st = O_SINF(theta);
    return normalize3(f3(st * O_COSF(phi), O_COSF(theta), st * O_SINF(phi)));
}
static inline OF3 o_envTex(const OScene* s, float u, float v)
{
    OF4 t = o_tex2d_f4(s->envTexels, s->envW, s->envH, 0, u, v);
    return f3(t.x * s->envIntensity, t.y * s->envIntensity, t.z * s->envIntensity);
}
static OF3 o_envEval(const OScene* s, OF3 dir)
{
    OF2 uv = o_dirToEquirect(dir, s->envRotation);
    return o_envTex(s, uv.x, uv.y);
}
static inline int o_cdfSearch(const float* cdf, int count, float x)
{
    int lo = 0, hi = count;
    while (lo + 1 < hi) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}
/* solid-angle pdf from a discrete pixel probability (rt_env_map.cuh:122-131) */
static inline float o_envSolidAngle(const OScene* s, float pPix, float v)
{
    const float theta = v * O_MPI;
    const float st = fmaxf(O_SINF(theta), 1e-6f);
    return (pPix * (float)s->envW * (float)s->envH) / (2.0f * O_MPI * O_MPI * st);
}
static float o_envPdf(const OScene* s, OF3 dir)
{
    if (s->envTotalPower <= 0.0f) return 0.0f;
    OF2 uv = o_dirToEquirect(dir, s->envRotation);
    float fx = uv.x * (float)s->envW;
    float fy = uv.y * (float)s->envH;
    int ix = (int)fx; ix = ix < 0 ? 0 : ix; ix = ix > s->envW - 1 ? s->envW - 1 : ix;
    int iy = (int)fy; iy = iy < 0 ? 0 : iy; iy = iy > s->envH - 1 ? s->envH - 1 : iy;
    if (s->envSampling == O_ENV_ALIAS) {
        const float p = s->envPixelPdf[(size_t)iy * s->envW + ix];
        if (p <= 0.0f) return 0.0f;
        return o_envSolidAngle(s, p, uv.y);
    }
    const float msum = s->envMarginal[s->envH];
    const float rw = s->envMarginal[iy + 1] - s->envMarginal[iy];
    if (msum <= 0.0f || rw <= 0.0f) return 0.0f;
    const float pRow = rw / msum;
    const float* row = s->envConditional + (size_t)iy * (s->envW + 1);
    const float rsum = row[s->envW];
    const float cw = row[ix + 1] - row[ix];
    if (rsum <= 0.0f || cw <= 0.0f) return 0.0f;
    const float pCol = cw / rsum;
    const float theta = uv.y * O_MPI;
    const float st = fmaxf(O_SINF(theta), 1e-6f);
    return (pRow * pCol * (float)s->envW * (float)s->envH) / (2.0f * O_MPI * O_MPI * st);
}

typedef struct { OF3 dir; float pdf; OF3 rad; } OEnvSample;

/* Alias-table pick: index from u, coin and continuous remainder from the
 * fractional part.  Shared by the row and column levels. */
static inline int o_aliasPick(const float* prob, const int* alias, int n, float u, float* frac)
{
    float x = u * (float)n;
    int i = (int)x;
    if (i > n - 1) i = n - 1;
    float f = x - (float)i;
    const float p = prob[i];
    if (f < p) {
        *frac = f / p;
        return i;
    }
    *frac = (f - p) / (1.0f - p);
    return alias[i];
}

static OEnvSample o_envSample(const OScene* s, float u0, float u1)
{
    OEnvSample r;
    r.dir = f3(0.0f, 1.0f, 0.0f); r.pdf = 0.0f; r.rad = f3(0, 0, 0);
    if (s->envTotalPower <= 0.0f) return r;
    if (s->envSampling == O_ENV_ALIAS) {
        float fr, fc;
        const int row = o_aliasPick(s->aliasRowProb, s->aliasRowIdx, s->envH, u0, &fr);
        const int col = o_aliasPick(s->aliasColProb + (size_t)row * s->envW, s->aliasColIdx + (size_t)row * s->envW,
                                    s->envW, u1, &fc);
        if (fr >= 1.0f) fr = 0x1.fffffep-1f;
        if (fc >= 1.0f) fc = 0x1.fffffep-1f;
        float u = ((float)col + fc) / (float)s->envW;
        float v = ((float)row + fr) / (float)s->envH;
        r.dir = o_equirectToDir(u, v, s->envRotation);
        r.rad = o_envTex(s, u, v);
        const float p = s->envPixelPdf[(size_t)row * s->envW + col];
        r.pdf = (p > 0.0f) ? o_envSolidAngle(s, p, v) : 0.0f;
        return r;
    }
    const float msum = s->envMarginal[s->envH];
    if (msum <= 0.0f) return r;
    const float xr = u0 * msum;
    const int row = o_cdfSearch(s->envMarginal, s->envH, xr);
    const float c0r = s->envMarginal[row], c1r = s->envMarginal[row + 1];
    const float dRow = c1r - c0r;
    float fracRow = (dRow > 0.0f) ? (xr - c0r) / dRow : 0.0f;
    const float* rc = s->envConditional + (size_t)row * (s->envW + 1);
    const float rsum = rc[s->envW];
    if (rsum <= 0.0f) return r;
    const float xc = u1 * rsum;
    const int col = o_cdfSearch(rc, s->envW, xc);
    const float c0c = rc[col], c1c = rc[col + 1];
    const float dCol = c1c - c0c;
    float fracCol = (dCol > 0.0f) ? (xc - c0c) / dCol : 0.0f;
    float u = ((float)col + fracCol) / (float)s->envW;
    float v = ((float)row + fracRow) / (float)s->envH;
    r.dir = o_equirectToDir(u, v, s->envRotation);
    r.rad = o_envTex(s, u, v);
    const float pRow = dRow / msum, pCol = dCol / rsum;
    const float theta = v * O_MPI;
    const float st = fmaxf(O_SINF(theta), 1e-6f);
    r.pdf = (pRow * pCol * (float)s->envW * (float)s->envH) / (2.0f * O_MPI * O_MPI * st);
    return r;
}

/* Host CDF build: src/host/scene_upload.cu:422-459 (FP32, sequential). */
void or_env_build_cdf(const float* rgba, int w, int h, float* marg, float* cond, float* totalPower)
{
    const float PI = 3.14159265358979323846f;
    marg[0] = 0.0f;
    for (int iy = 0; iy < h; ++iy) {
        const float theta = PI * ((float)iy + 0.5f) / (float)h;
        const float st = sinf(theta);   /* the reference computes this on the host with std::sin */
        float* row = cond + (size_t)iy * (w + 1);
        row[0] = 0.0f;
        for (int ix = 0; ix < w; ++ix) {
            const size_t pb = ((size_t)iy * w + ix) * 4;
            const float lum = 0.2126f * rgba[pb] + 0.7152f * rgba[pb + 1] + 0.0722f * rgba[pb + 2];
            row[ix + 1] = row[ix] + lum * st;
        }
        marg[iy + 1] = marg[iy] + row[w];
    }
    *totalPower = marg[h];
}

/* Vose's alias method (M. D. Vose, IEEE TSE 17(9), 1991) over weights w[0..n)
 * with FP64 arithmetic.  Deterministic work-list discipline: both lists are
 * filled in ascending index order and consumed from the end (stacks). */
static void o_vose(const double* w, int n, double sum, float* prob, int* alias, int* small, int* large, double* scaled)
{
    int ns = 0, nl = 0;
    if (!(sum > 0.0)) {
        for (int i = 0; i < n; ++i) { prob[i] = 1.0f; alias[i] = i; }
        return;
    }
    for (int i = 0; i < n; ++i) {
        scaled[i] = w[i] * (double)n / sum;
        if (scaled[i] < 1.0) small[ns++] = i; else large[nl++] = i;
    }
    while (ns > 0 && nl > 0) {
        const int l = small[--ns];
        const int g = large[--nl];
        prob[l] = (float)scaled[l];
        alias[l] = g;
        scaled[g] = (scaled[g] + scaled[l]) - 1.0;
        if (scaled[g] < 1.0) small[ns++] = g; else large[nl++] = g;
    }
    while (nl > 0) { const int g = large[--nl]; prob[g] = 1.0f; alias[g] = g; }
    while (ns > 0) { const int l = small[--ns]; prob[l] = 1.0f; alias[l] = l; }
}

/* FP64 two-level alias tables + per-pixel discrete pdf (fast sampling mode). */
void or_env_build_alias(const float* rgba, int w, int h, float* rowProb, int* rowIdx, float* colProb, int* colIdx,
                        float* pixelPdf, double* totalPowerD)
{
    double* wt = (double*)malloc(sizeof(double) * (size_t)w * h);
    double* rowSum = (double*)malloc(sizeof(double) * h);
    int* small = (int*)malloc(sizeof(int) * (size_t)(w > h ? w : h));
    int* large = (int*)malloc(sizeof(int) * (size_t)(w > h ? w : h));
    double* scaled = (double*)malloc(sizeof(double) * (size_t)(w > h ? w : h));
    double total = 0.0;
    for (int iy = 0; iy < h; ++iy) {
        const double theta = OM_PI_D * ((double)iy + 0.5) / (double)h;
        const double st = om_sin_d(theta);
        double rs = 0.0;
        for (int ix = 0; ix < w; ++ix) {
            const size_t pb = ((size_t)iy * w + ix) * 4;
            const double lum = 0.2126 * (double)rgba[pb] + 0.7152 * (double)rgba[pb + 1] + 0.0722 * (double)rgba[pb + 2];
            const double v = lum * st;
            wt[(size_t)iy * w + ix] = v;
            rs += v;
        }
        rowSum[iy] = rs;
        total += rs;
    }
    for (int iy = 0; iy < h; ++iy) {
        o_vose(wt + (size_t)iy * w, w, rowSum[iy], colProb + (size_t)iy * w, colIdx + (size_t)iy * w, small, large, scaled);
        for (int ix = 0; ix < w; ++ix)
            pixelPdf[(size_t)iy * w + ix] = (total > 0.0) ? (float)(wt[(size_t)iy * w + ix] / total) : 0.0f;
    }
    o_vose(rowSum, h, total, rowProb, rowIdx, small, large, scaled);
    *totalPowerD = total;
    free(wt); free(rowSum); free(small); free(large); free(scaled);
}

void or_env_eval(const OScene* s, const float* dirs, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        OF3 r = o_envEval(s, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
}
void or_env_pdf(const OScene* s, const float* dirs, float* out, int n)
{
    for (int i = 0; i < n; ++i) out[i] = o_envPdf(s, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
}
void or_env_sample(const OScene* s, const float* u, float* outDir, float* outPdf, float* outRad, int n)
{
    for (int i = 0; i < n; ++i) {
        OEnvSample r = o_envSample(s, u[2 * i], u[2 * i + 1]);
        outDir[3 * i] = r.dir.x; outDir[3 * i + 1] = r.dir.y; outDir[3 * i + 2] = r.dir.z;
        outPdf[i] = r.pdf;
        outRad[3 * i] = r.rad.x; outRad[3 * i + 1] = r.rad.y; outRad[3 * i + 2] = r.rad.z;
    }
}

/* ------------------------------------------------------------------ */
/* emitter sampling -- rt_emitter_sampling.cuh:33-224                 */
/* ------------------------------------------------------------------ */
typedef struct { OF3 origin, hitPoint, hitNormal; float pdf, emitterPdf; OF3 dirToLight; } OEQ;

static int o_sampleCdfReuse(const float* cdf, int count, float* u, float* outPdf)
{
    const float sum = cdf[count];
    if (sum <= 0.0f || count <= 0) { *outPdf = 0.0f; *u = 0.0f; return 0; }
    float x = *u * sum;
    int lo = 0, hi = count;
    while (lo + 1 < hi) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] <= x) lo = mid;
        else hi = mid;
    }
    int idx = lo;
    float c0 = cdf[idx], c1 = cdf[idx + 1];
    float den = c1 - c0;
    if (den <= 0.0f) { *u = 0.0f; *outPdf = 0.0f; return idx; }
    *u = (x - c0) / den;
    *outPdf = den / sum;
    return idx;
}

static inline OF3 o_checkRadiance(OF3 rad, const OEQ* q)
{
    const OF3 neg = f3(-q->dirToLight.x, -q->dirToLight.y, -q->dirToLight.z);
    const float c = dot3(q->hitNormal, neg);
    if (c <= 0.0f) return f3(0, 0, 0);
    return rad;
}

static int o_findEmitter(const OScene* s, int tri)
{
    if (!s->emitters || !s->emitterTriIndices || s->emitterCount <= 0 || tri < 0) return -1;
    for (int e = 0; e < s->emitterCount; ++e) {
        const OEmitter* E = &s->emitters[e];
        for (int j = 0; j < E->triCount; ++j)
            if (s->emitterTriIndices[E->triIndexOffset + j] == tri) return e;
    }
    return -1;
}
static float o_sceneEmitterPdf(const OScene* s, int e)
{
    if (e < 0 || s->emitterCount <= 0 || !s->sceneEmitterCdf) return 0.0f;
    const float sum = s->sceneEmitterCdf[s->emitterCount];
    if (sum <= 0.0f) return 0.0f;
    const float w = s->sceneEmitterCdf[e + 1] - s->sceneEmitterCdf[e];
    return w / sum;
}

static OF3 o_sampleGenerator(const OScene* s, OEQ* q, float u0, float u1)
{
    q->emitterPdf = 0.0f;
    if (s->emitterCount <= 0) return f3(0, 0, 0);
    /* sampleRandomEmitter :304-329 */
    float epdf = 0.0f;
    const int e = o_sampleCdfReuse(s->sceneEmitterCdf, s->emitterCount, &u0, &epdf);
    const OEmitter E = s->emitters[e];
    /* sampleMeshEmitter :172-205 */
    OF3 pos = f3(0, 0, 0), nrm = f3(0, 0, 0);
    float mpdf = 0.0f;
    if (E.triCount > 0) {
        const float* tcdf = s->emitterTriCdf + E.cdfOffset;
        float tp = 0.0f;
        const int li = o_sampleCdfReuse(tcdf, E.triCount, &u0, &tp);
        const int ti = s->emitterTriIndices[E.triIndexOffset + li];
        const OTri T = s->triangles[ti];
        float root = sqrtf(fmaxf(0.0f, 1.0f - u0));
        float al = 1.0f - root;
        float be = u1 * root;
        float ga = 1.0f - al - be;
        pos = add3(add3(mul3s(T.v0, al), mul3s(T.v1, be)), mul3s(T.v2, ga));
        nrm = normalize3(cross3(sub3(T.v1, T.v0), sub3(T.v2, T.v0)));
        const float area = tcdf[E.triCount];
        if (area > 0.0f) mpdf = 1.0f / area;
    }
    /* sampleGenerator :280-302 */
    q->hitPoint = pos;
    q->hitNormal = nrm;
    q->pdf = mpdf;
    q->dirToLight = normalize3(sub3(q->hitPoint, q->origin));
    q->emitterPdf = epdf;
    return o_checkRadiance(E.radiance, q);
}

/* ------------------------------------------------------------------ */
/* path state, direct lighting, integrator                            */
/* ------------------------------------------------------------------ */
typedef struct {
    OF3 o, d;           /* ray */
    OF3 tp, L;          /* throughput, accumulated colour */
    int bounce;
    float eta, brdfPdf;
    int specular;
} OPath;

typedef struct { OF3 p, n; OF2 uv; int tri; } OHit;
typedef struct { OF3 o, d; float tmax; OF3 c; } OShadow;

/* rt_direct_lighting.cuh:36-49 */
static inline float o_areaToSolid(float pA, const OEQ* q)
{
    const OF3 diff = sub3(q->hitPoint, q->origin);
    const float d2 = dot3(diff, diff);
    const OF3 neg = f3(-q->dirToLight.x, -q->dirToLight.y, -q->dirToLight.z);
    const float den = fmaxf(fabsf(dot3(q->hitNormal, neg)), 1e-3f);
    return pA * d2 / den;
}
/* :60-99 */
static void o_accumulateEmitterHit(const OScene* s, OPath* p, const OHit* h)
{
    const OF3 rad0 = s->emission[h->tri];
    OEQ q; memset(&q, 0, sizeof q);
    q.origin = p->o; q.hitPoint = h->p; q.hitNormal = h->n; q.dirToLight = p->d;
    float w = 1.0f;
    if (!p->specular) {
        const int e = o_findEmitter(s, h->tri);
        if (e >= 0) {
            const float ap = (s->emitters[e].areaSum <= 0.0f) ? 0.0f : 1.0f / s->emitters[e].areaSum;
            const float pA = ap * o_sceneEmitterPdf(s, e);
            const float pS = o_areaToSolid(pA, &q);
            const float den = p->brdfPdf + pS;
            if (den <= 0.0f) w = 0.0f;
            else w = p->brdfPdf / den;
        }
    }
    const OF3 rad = o_checkRadiance(rad0, &q);
    p->L = add3(p->L, mul3s(mul3v(rad, p->tp), w));
}
/* :107-164 */
static int o_prepareArea(const OScene* s, OPath* p, uint32_t* rng, const OHit* h, const OBsdf* b, OShadow* sr)
{
    const float ul0 = rngNextFloat01(rng);
    const float ul1 = rngNextFloat01(rng);
    OEQ q; memset(&q, 0, sizeof q);
    q.origin = h->p;
    OF3 le = o_sampleGenerator(s, &q, ul0, ul1);
    if ((le.x <= 0.0f && le.y <= 0.0f && le.z <= 0.0f) || q.emitterPdf <= 0.0f || q.pdf <= 0.0f) return 0;
    const float dist = distance3(q.hitPoint, h->p);
    const float geo = fabsf(dot3(h->n, q.dirToLight)) * fabsf(dot3(q.hitNormal, mul3s(q.dirToLight, -1.0f))) /
                      (dist * dist);
    OBRec r; memset(&r, 0, sizeof r);
    r.wi = toLocalN(h->n, mul3s(p->d, -1.0f));
    r.wo = toLocalN(h->n, q.dirToLight);
    r.measure = O_ESOLID;
    const OF3 fr = o_bsdfEval(b, &r);
    const float pA = q.emitterPdf * q.pdf;
    const float pS = o_areaToSolid(pA, &q);
    const float pB = o_bsdfPdf(b, &r);
    const float den = pB + pS;
    if (den <= 0.0f) return 0;
    const float lw = pS / den;
    OF3 c = mul3v(fr, le);
    c = mul3s(c, lw);
    c = mul3s(c, geo);
    c = div3(c, pA);
    sr->o = h->p; sr->d = q.dirToLight; sr->tmax = dist - O_RT_EPSILON; sr->c = mul3v(c, p->tp);
    return 1;
}
/* :175-230 */
static int o_prepareSpot(const OScene* s, const OPath* p, const OHit* h, const OBsdf* b, int si, OShadow* sr)
{
    const OSpot sp = s->spots[si];
    const OF3 o2l = sub3(sp.position, h->p);
    const float sq = dot3(o2l, o2l);
    if (sq < O_RT_EPSILON * O_RT_EPSILON) return 0;
    const float dist = sqrtf(sq);
    const OF3 dl = div3(o2l, dist);
    const float lc = dot3(mul3s(dl, -1.0f), sp.direction);
    OF3 le;
    if (lc <= sp.outerConeCosine) return 0;
    else if (lc >= sp.innerConeCosine) le = mul3s(sp.radiance, sp.intensity / sq);
    else {
        float fo = (lc - sp.outerConeCosine) / (sp.innerConeCosine - sp.outerConeCosine);
        float sm = (fo * fo) * (3.0f - (2.0f * fo));
        le = mul3s(sp.radiance, (sp.intensity * sm) / sq);
    }
    OBRec r; memset(&r, 0, sizeof r);
    r.wi = toLocalN(h->n, mul3s(p->d, -1.0f));
    r.wo = toLocalN(h->n, dl);
    r.measure = O_ESOLID;
    const OF3 fr = o_bsdfEval(b, &r);
    const float cs = fabsf(dot3(h->n, dl));
    sr->o = h->p; sr->d = dl; sr->tmax = dist - O_RT_EPSILON;
    sr->c = mul3v(mul3s(mul3v(fr, le), cs), p->tp);
    return 1;
}
/* :237-259 */
static void o_accumulateEnvHit(const OScene* s, OPath* p)
{
    if (!s->hasEnv) return;
    const OF3 er = o_envEval(s, p->d);
    float w = 1.0f;
    if (!p->specular) {
        const float ep = o_envPdf(s, p->d);
        const float sum = p->brdfPdf + ep;
        if (sum > 0.0f) w = p->brdfPdf / sum;
        else w = 0.0f;
    }
    p->L = add3(p->L, mul3s(mul3v(er, p->tp), w));
}
/* :267-315 */
static int o_prepareEnv(const OScene* s, OPath* p, uint32_t* rng, const OHit* h, const OBsdf* b, OShadow* sr)
{
    if (!s->hasEnv) return 0;
    const float u0 = rngNextFloat01(rng);
    const float u1 = rngNextFloat01(rng);
    OEnvSample es = o_envSample(s, u0, u1);
    if (es.pdf <= 0.0f) return 0;
    if (es.rad.x <= 0.0f && es.rad.y <= 0.0f && es.rad.z <= 0.0f) return 0;
    const float ca = dot3(h->n, es.dir);
    if (ca <= 0.0f) return 0;
    OBRec r; memset(&r, 0, sizeof r);
    r.wi = toLocalN(h->n, mul3s(p->d, -1.0f));
    r.wo = toLocalN(h->n, es.dir);
    r.measure = O_ESOLID;
    const OF3 fr = o_bsdfEval(b, &r);
    const float bp = o_bsdfPdf(b, &r);
    const float sum = bp + es.pdf;
    if (sum <= 0.0f) return 0;
    const float lw = es.pdf / sum;
    OF3 c = mul3v(fr, es.rad);
    c = mul3s(c, ca);
    c = div3(c, es.pdf);
    c = mul3s(c, lw);
    sr->o = h->p; sr->d = es.dir; sr->tmax = 1e30f - O_RT_EPSILON; sr->c = mul3v(c, p->tp);
    return 1;
}
/* rt_path_integrator.cuh:25-47 */
static void o_scatter(OPath* p, uint32_t* rng, const OHit* h, const OBsdf* b)
{
    OBRec r; memset(&r, 0, sizeof r);
    r.wi = toLocalN(h->n, mul3s(p->d, -1.0f));
    r.rndExtra = rngNextFloat01(rng);
    const float u0 = rngNextFloat01(rng);
    const float u1 = rngNextFloat01(rng);
    OF3 sw = o_bsdfSample(b, &r, u0, u1);
    p->brdfPdf = o_bsdfPdf(b, &r);
    const OF3 bd = normalize3(toWorldN(h->n, r.wo));
    p->o = add3(h->p, mul3s(bd, O_RT_EPSILON));
    p->d = bd;
    p->tp = mul3v(p->tp, sw);
    p->eta *= r.eta;
}
/* :54-65 */
static int o_roulette(OPath* p, uint32_t* rng, int rrStart)
{
    if (p->bounce > rrStart) {
        const float cp = fminf(maxCoeff3(p->tp) * p->eta * p->eta, 0.99f);
        if (rngNextFloat01(rng) >= cp) return 0;
        p->tp = div3(p->tp, cp);
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* camera -- rt_camera.cuh:15-37                                      */
/* ------------------------------------------------------------------ */
static void o_primaryRay(int px, int py, int w, int h, const OCamera* c, float jx, float jy, OF3* o, OF3* d)
{
    const float fx = ((float)px + 0.5f + jx) / (float)w;
    const float fy = ((float)py + 0.5f + jy) / (float)h;
    const float ndcX = 2.0f * fx - 1.0f;
    const float ndcY = 2.0f * fy - 1.0f;
    const float th = O_TANF(0.5f * c->fovYRadians);
    const float sx = ndcX * c->aspect * th;
    const float sy = ndcY * th;
    OF3 dir = add3(c->forward, add3(mul3s(c->right, sx), mul3s(c->up, sy)));
    *o = c->origin;
    *d = normalize3(dir);
}

/* ------------------------------------------------------------------ */
/* traversal: watertight triangle test + CPU BVH                      */
/* ------------------------------------------------------------------ */
typedef struct {
    OF3 o;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    int valid;
} ORayPre;

static inline float o_comp(OF3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

static ORayPre o_rayPre(OF3 o, OF3 d)
{
    ORayPre r;
    r.o = o;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    if (ay > ax) kz = 1;
    if (az > (kz == 0 ? ax : ay)) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dz = o_comp(d, kz);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.valid = (dz != 0.0f) && (dz == dz);
    r.Sx = o_comp(d, kx) / dz;
    r.Sy = o_comp(d, ky) / dz;
    r.Sz = 1.0f / dz;
    return r;
}

/* Returns 1 on a hit with t in [tmin, tmax]; writes t, u (weight of v1), v (weight of v2). */
static int o_isectTri(const ORayPre* r, const OTri* T, float tmin, float tmax, float* ot, float* ou, float* ov)
{
    const OF3 A = sub3(T->v0, r->o), B = sub3(T->v1, r->o), C = sub3(T->v2, r->o);
    const float Akz = o_comp(A, r->kz), Bkz = o_comp(B, r->kz), Ckz = o_comp(C, r->kz);
    const float Ax = o_comp(A, r->kx) - r->Sx * Akz;
    const float Ay = o_comp(A, r->ky) - r->Sy * Akz;
    const float Bx = o_comp(B, r->kx) - r->Sx * Bkz;
    const float By = o_comp(B, r->ky) - r->Sy * Bkz;
    const float Cx = o_comp(C, r->kx) - r->Sx * Ckz;
    const float Cy = o_comp(C, r->ky) - r->Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
    const float det = U + V + W;
    if (det == 0.0f) return 0;
    const float Az = r->Sz * Akz, Bz = r->Sz * Bkz, Cz = r->Sz * Ckz;
    const float Tn = U * Az + V * Bz + W * Cz;
    const float t = Tn / det;
    if (!(t >= tmin && t <= tmax)) return 0;
    *ot = t;
    *ou = V / det;
    *ov = W / det;
    return 1;
}

/* ---- CPU BVH (binary, object-median split on the longest centroid axis) ---- */
typedef struct { float lo[3], hi[3]; int left, right; int first, count; } OBvhNode;
typedef struct { OBvhNode* nodes; int nodeCount; int* idx; double maxAbs; } OAccel;

static void o_triBounds(const OTri* t, float lo[3], float hi[3])
{
    lo[0] = fminf(t->v0.x, fminf(t->v1.x, t->v2.x)); hi[0] = fmaxf(t->v0.x, fmaxf(t->v1.x, t->v2.x));
    lo[1] = fminf(t->v0.y, fminf(t->v1.y, t->v2.y)); hi[1] = fmaxf(t->v0.y, fmaxf(t->v1.y, t->v2.y));
    lo[2] = fminf(t->v0.z, fminf(t->v1.z, t->v2.z)); hi[2] = fmaxf(t->v0.z, fmaxf(t->v1.z, t->v2.z));
}

typedef struct { const OTri* tris; float* cen; int axis; } OSortCtx;
static OSortCtx g_sortCtx;   /* qsort has no context argument; builds are single-threaded */
static int o_cmpCen(const void* a, const void* b)
{
    const int ia = *(const int*)a, ib = *(const int*)b;
    const float ca = g_sortCtx.cen[3 * ia + g_sortCtx.axis], cb = g_sortCtx.cen[3 * ib + g_sortCtx.axis];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
    return (ia < ib) ? -1 : (ia > ib);
}

static int o_buildRec(OAccel* A, const OTri* tris, float* cen, int first, int count)
{
    const int ni = A->nodeCount++;
    OBvhNode* n = &A->nodes[ni];
    n->lo[0] = n->lo[1] = n->lo[2] = FLT_MAX;
    n->hi[0] = n->hi[1] = n->hi[2] = -FLT_MAX;
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = first; i < first + count; ++i) {
        float lo[3], hi[3];
        o_triBounds(&tris[A->idx[i]], lo, hi);
        for (int k = 0; k < 3; ++k) {
            n->lo[k] = fminf(n->lo[k], lo[k]); n->hi[k] = fmaxf(n->hi[k], hi[k]);
            const float c = cen[3 * A->idx[i] + k];
            clo[k] = fminf(clo[k], c); chi[k] = fmaxf(chi[k], c);
        }
    }
    if (count <= 4) { n->left = n->right = -1; n->first = first; n->count = count; return ni; }
    int axis = 0;
    if (chi[1] - clo[1] > chi[axis] - clo[axis]) axis = 1;
    if (chi[2] - clo[2] > chi[axis] - clo[axis]) axis = 2;
    g_sortCtx.cen = cen; g_sortCtx.axis = axis;
    qsort(A->idx + first, (size_t)count, sizeof(int), o_cmpCen);
    const int half = count / 2;
    const int l = o_buildRec(A, tris, cen, first, half);
    const int r = o_buildRec(A, tris, cen, first + half, count - half);
    n = &A->nodes[ni];
    n->left = l; n->right = r; n->first = 0; n->count = 0;
    return ni;
}

int or_build_accel(OScene* s)
{
    or_free_accel(s);
    const int T = s->triangleCount;
    if (T <= 0) return 0;
    OAccel* A = (OAccel*)calloc(1, sizeof(OAccel));
    A->nodes = (OBvhNode*)malloc(sizeof(OBvhNode) * (size_t)(2 * T + 1));
    A->idx = (int*)malloc(sizeof(int) * (size_t)T);
    float* cen = (float*)malloc(sizeof(float) * 3 * (size_t)T);
    double ext = 0.0;
    for (int i = 0; i < T; ++i) {
        A->idx[i] = i;
        float lo[3], hi[3];
        o_triBounds(&s->triangles[i], lo, hi);
        for (int k = 0; k < 3; ++k) {
            cen[3 * i + k] = 0.5f * (lo[k] + hi[k]);
            ext = fmax(ext, fmax(fabs((double)lo[k]), fabs((double)hi[k])));
        }
    }
    A->maxAbs = ext;
    o_buildRec(A, s->triangles, cen, 0, T);
    free(cen);
    s->accel = A;
    return 0;
}

void or_free_accel(OScene* s)
{
    if (!s->accel) return;
    OAccel* A = (OAccel*)s->accel;
    free(A->nodes); free(A->idx); free(A);
    s->accel = NULL;
}

/* Conservative slab test in double, each slab widened by the bound on the
 * watertight test's t error (128 * 2^-24 * (max|origin| + max|scene coordinate|)). */
static inline int o_boxHit(const OAccel* A, const OBvhNode* n, const double o[3], const double inv[3],
                           double tmin, double tmax)
{
    double t0 = tmin, t1 = tmax;
    const double pad = 128.0 * 5.9604644775390625e-8 * (fmax(fabs(o[0]), fmax(fabs(o[1]), fabs(o[2]))) + A->maxAbs);
    (void)A;
    for (int k = 0; k < 3; ++k) {
        const double lo = (double)n->lo[k] - pad, hi = (double)n->hi[k] + pad;
        double a = (lo - o[k]) * inv[k], b = (hi - o[k]) * inv[k];
        if (a != a) a = -INFINITY;   /* 0 * inf when the origin lies on the slab plane */
        if (b != b) b = INFINITY;
        if (a > b) { const double t = a; a = b; b = t; }
        if (a > t0) t0 = a;
        if (b < t1) t1 = b;
    }
    return t0 <= t1 * (1.0 + 1e-9);
}

/* closest hit; ties in t resolved to the lower triangle index */
static int o_traceClosest(const OScene* s, OF3 o, OF3 d, float tmin, float tmax, float* tOut, float* uOut, float* vOut)
{
    const ORayPre rp = o_rayPre(o, d);
    if (!rp.valid) return -1;
    int best = -1;
    float bt = tmax, bu = 0.0f, bv = 0.0f;
    const OAccel* A = (const OAccel*)s->accel;
    if (!A) {
        for (int i = 0; i < s->triangleCount; ++i) {
            float t, u, v;
            if (o_isectTri(&rp, &s->triangles[i], tmin, bt, &t, &u, &v)) {
                if (best < 0 || t < bt || (t == bt && i < best)) { best = i; bt = t; bu = u; bv = v; }
            }
        }
    } else {
        const double od[3] = {o.x, o.y, o.z};
        const double inv[3] = {1.0 / (double)d.x, 1.0 / (double)d.y, 1.0 / (double)d.z};
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const OBvhNode* n = &A->nodes[stack[--sp]];
            if (!o_boxHit(A, n, od, inv, (double)tmin, (double)bt * (1.0 + 1e-6) + 1e-30)) continue;
            if (n->count > 0) {
                for (int j = n->first; j < n->first + n->count; ++j) {
                    const int i = A->idx[j];
                    float t, u, v;
                    if (o_isectTri(&rp, &s->triangles[i], tmin, bt, &t, &u, &v)) {
                        if (best < 0 || t < bt || (t == bt && i < best)) { best = i; bt = t; bu = u; bv = v; }
                    }
                }
            } else {
                stack[sp++] = n->left;
                stack[sp++] = n->right;
            }
        }
    }
    if (best >= 0) { *tOut = bt; *uOut = bu; *vOut = bv; }
    return best;
}

static int o_traceOccluded(const OScene* s, OF3 o, OF3 d, float tmin, float tmax)
{
    const ORayPre rp = o_rayPre(o, d);
    if (!rp.valid) return 0;
    const OAccel* A = (const OAccel*)s->accel;
    float t, u, v;
    if (!A) {
        for (int i = 0; i < s->triangleCount; ++i)
            if (o_isectTri(&rp, &s->triangles[i], tmin, tmax, &t, &u, &v)) return 1;
        return 0;
    }
    const double od[3] = {o.x, o.y, o.z};
    const double inv[3] = {1.0 / (double)d.x, 1.0 / (double)d.y, 1.0 / (double)d.z};
    int stack[128]; int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const OBvhNode* n = &A->nodes[stack[--sp]];
        if (!o_boxHit(A, n, od, inv, (double)tmin, (double)tmax * (1.0 + 1e-6) + 1e-30)) continue;
        if (n->count > 0) {
            for (int j = n->first; j < n->first + n->count; ++j)
                if (o_isectTri(&rp, &s->triangles[A->idx[j]], tmin, tmax, &t, &u, &v)) return 1;
        } else {
            stack[sp++] = n->left;
            stack[sp++] = n->right;
        }
    }
    return 0;
}

void or_trace_closest(const OScene* s, const float* rays, int n, int* outTri, float* outTuv)
{
    for (int i = 0; i < n; ++i) {
        float t = 0, u = 0, v = 0;
        const int tri = o_traceClosest(s, f3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]),
                                       f3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]), O_RT_EPSILON, 1e30f,
                                       &t, &u, &v);
        outTri[i] = tri;
        outTuv[3 * i] = t; outTuv[3 * i + 1] = u; outTuv[3 * i + 2] = v;
    }
}

void or_trace_occluded(const OScene* s, const float* rays, const float* tmax, int n, uint8_t* outOcc)
{
    for (int i = 0; i < n; ++i)
        outOcc[i] = (uint8_t)o_traceOccluded(s, f3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]),
                                             f3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]), O_RT_EPSILON,
                                             tmax[i]);
}

/* closest-hit attribute interpolation: src/optix_programs.cu:110-141 */
static void o_fillHit(const OScene* s, OF3 o, OF3 d, int tri, float t, float u, float v, OHit* h)
{
    const OTri* T = &s->triangles[tri];
    const float w0 = 1.0f - u - v;
    h->tri = tri;
    h->p = f3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    h->n = normalize3(f3(w0 * T->n0.x + u * T->n1.x + v * T->n2.x, w0 * T->n0.y + u * T->n1.y + v * T->n2.y,
                         w0 * T->n0.z + u * T->n1.z + v * T->n2.z));
    h->uv.x = w0 * T->uv0.x + u * T->uv1.x + v * T->uv2.x;
    h->uv.y = w0 * T->uv0.y + u * T->uv1.y + v * T->uv2.y;
}

/* ------------------------------------------------------------------ */
/* one sample: src/wavefront/ray_generate.cu:42-80 + the bounce loop   */
/* (src/host/wavefront_host.cu:171-222, ray_shade.cu:103-183) in the   */
/* megakernel's per-path order (src/optix_programs.cu:54-108).         */
/* ------------------------------------------------------------------ */
static OF3 o_renderSample(const OScene* s, const OCamera* cam, const OConfig* cfg, uint32_t pixel, uint32_t sampleIndex,
                          int* hitLog, OStats* st, float* rayLog, uint32_t* rngIO)
{
    const int px = (int)(pixel % (uint32_t)cfg->width);
    const int py = (int)(pixel / (uint32_t)cfg->width);
    /* rngIO: a stream carried from the previous path of the pixel (megakernel), updated on return */
    uint32_t rng = rngIO ? *rngIO : rngMake(or_hash_uint(pixel ^ (sampleIndex * 0x9e3779b9u)));
    const float jx = rngNextFloat01(&rng) - 0.5f;
    const float jy = rngNextFloat01(&rng) - 0.5f;
    OPath p;
    o_primaryRay(px, py, cfg->width, cfg->height, cam, jx, jy, &p.o, &p.d);
    p.tp = f3(1.f, 1.f, 1.f);
    p.L = f3(0.f, 0.f, 0.f);
    p.eta = 1.f;
    p.brdfPdf = 0.f;
    p.specular = 1;
    p.bounce = 0;
    if (hitLog) for (int i = 0; i < cfg->maxDepth; ++i) hitLog[i] = -2;

    for (int bounce = 0; bounce < cfg->maxDepth; ++bounce) {
        float t, u, v;
        if (rayLog) {
            float* r6 = rayLog + 6 * bounce;
            r6[0] = p.o.x; r6[1] = p.o.y; r6[2] = p.o.z; r6[3] = p.d.x; r6[4] = p.d.y; r6[5] = p.d.z;
        }
        const int tri = o_traceClosest(s, p.o, p.d, O_RT_EPSILON, 1e30f, &t, &u, &v);
        if (st) st->extends++;
        if (hitLog) hitLog[bounce] = tri;
        if (tri < 0) {
            o_accumulateEnvHit(s, &p);
            break;
        }
        OHit h;
        o_fillHit(s, p.o, p.d, tri, t, u, v, &h);
        const OBsdf b = o_loadBsdf(s, tri, h.uv);
        if (s->emitterFlags[tri] != 0) o_accumulateEmitterHit(s, &p, &h);
        if (o_isDiffuseClass(&b)) {
            p.specular = 0;
            OShadow sr;
            if (o_prepareArea(s, &p, &rng, &h, &b, &sr)) {
                if (st) st->shadowRays++;
                if (!o_traceOccluded(s, sr.o, sr.d, O_RT_EPSILON, sr.tmax)) p.L = add3(p.L, sr.c);
            }
            for (int si = 0; si < s->spotCount; ++si) {
                if (o_prepareSpot(s, &p, &h, &b, si, &sr)) {
                    if (st) st->shadowRays++;
                    if (!o_traceOccluded(s, sr.o, sr.d, O_RT_EPSILON, sr.tmax)) p.L = add3(p.L, sr.c);
                }
            }
            if (o_prepareEnv(s, &p, &rng, &h, &b, &sr)) {
                if (st) st->shadowRays++;
                if (!o_traceOccluded(s, sr.o, sr.d, O_RT_EPSILON, sr.tmax)) p.L = add3(p.L, sr.c);
            }
        } else {
            p.specular = 1;
        }
        o_scatter(&p, &rng, &h, &b);
        if (!o_roulette(&p, &rng, cfg->rrStart)) break;
        p.bounce++;
    }
    if (rngIO) *rngIO = rng;
    return p.L;
}

void or_render_samples(const OScene* s, const OCamera* cam, const OConfig* cfg, const uint32_t* pixels,
                       const uint32_t* sampleIndices, int n, float* outRadiance, int* hitLog, OStats* stats,
                       int threads)
{
    int64_t ext = 0, sh = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) reduction(+ : ext, sh)
#endif
    for (int i = 0; i < n; ++i) {
        OStats local = {0, 0};
        OF3 L = o_renderSample(s, cam, cfg, pixels[i], sampleIndices[i], hitLog ? hitLog + (size_t)i * cfg->maxDepth : NULL,
                               &local, NULL, NULL);
        outRadiance[3 * i] = L.x; outRadiance[3 * i + 1] = L.y; outRadiance[3 * i + 2] = L.z;
        ext += local.extends; sh += local.shadowRays;
    }
    (void)threads;
    if (stats) { stats->extends += ext; stats->shadowRays += sh; }
}

/* per-bounce rays of one sample (diagnostics): rays [maxDepth*6], hits [maxDepth] */
void or_path_rays(const OScene* s, const OCamera* cam, const OConfig* cfg, uint32_t pixel, uint32_t sampleIndex,
                  float* rays, int* hits)
{
    for (int i = 0; i < 6 * cfg->maxDepth; ++i) rays[i] = NAN;
    (void)o_renderSample(s, cam, cfg, pixel, sampleIndex, hits, NULL, rays, NULL);
}

/* one megakernel frame, src/optix_programs.cu:54-108: per pixel one stream,
   makeRng(hashUint(pixel ^ frameIndex * 0x9e3779b9)), carried through spp
   paths in turn (each draws its jitter first); the paths' radiance summed in
   sample order from zero and scaled by 1/spp (div3, rt_cuda_math.cuh:28-33).
   Writes the frame's mean per pixel [n*3], the input of the Welford update. */
void or_render_megakernel(const OScene* s, const OCamera* cam, const OConfig* cfg, const uint32_t* pixels, int n,
                          uint32_t frameIndex, int spp, float* outMean, OStats* stats, int threads)
{
    int64_t ext = 0, sh = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) reduction(+ : ext, sh)
#endif
    for (int i = 0; i < n; ++i) {
        OStats local = {0, 0};
        uint32_t rng = rngMake(or_hash_uint(pixels[i] ^ (frameIndex * 0x9e3779b9u)));
        OF3 sum = f3(0.f, 0.f, 0.f);
        for (int k = 0; k < spp; ++k)
            sum = add3(sum, o_renderSample(s, cam, cfg, pixels[i], 0u, NULL, &local, NULL, &rng));
        const float inv = spp != 0 ? 1.0f / (float)spp : 0.0f;
        outMean[3 * i] = sum.x * inv; outMean[3 * i + 1] = sum.y * inv; outMean[3 * i + 2] = sum.z * inv;
        ext += local.extends; sh += local.shadowRays;
    }
    (void)threads;
    if (stats) { stats->extends += ext; stats->shadowRays += sh; }
}

/* ------------------------------------------------------------------ */
/* present -- rt_path_integrator.cuh:72-105                            */
/* ------------------------------------------------------------------ */
uint32_t or_pack_gamma(float r, float g, float b)
{
    float dr = O_POWF(fmaxf(0.0f, fminf(r, 1.0f)), 1.0f / 2.2f);
    float dg = O_POWF(fmaxf(0.0f, fminf(g, 1.0f)), 1.0f / 2.2f);
    float db = O_POWF(fmaxf(0.0f, fminf(b, 1.0f)), 1.0f / 2.2f);
    uint8_t R = (uint8_t)(dr * 255.0f), G = (uint8_t)(dg * 255.0f), B = (uint8_t)(db * 255.0f), A = 255;
    return ((uint32_t)A << 24) | ((uint32_t)B << 16) | ((uint32_t)G << 8) | R;
}

void or_present(float* accum, const float* radiance, int count, uint32_t frameIndex, uint32_t* outRGBA8)
{
    const float nf = (float)(frameIndex + 1);
    for (int i = 0; i < count; ++i) {
        float* a = accum + 3 * i;
        const float* x = radiance + 3 * i;
        a[0] = a[0] + (x[0] - a[0]) / nf;
        a[1] = a[1] + (x[1] - a[1]) / nf;
        a[2] = a[2] + (x[2] - a[2]) / nf;
        if (outRGBA8) outRGBA8[i] = or_pack_gamma(a[0], a[1], a[2]);
    }
}

/* ---- math entry points for accuracy tests ---- */
void or_math_eval(int fn, const float* a, const float* b, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        switch (fn) {
        case 0: out[i] = O_SINF(a[i]); break;
        case 1: out[i] = O_COSF(a[i]); break;
        case 2: out[i] = O_TANF(a[i]); break;
        case 3: out[i] = O_EXPF(a[i]); break;
        case 4: out[i] = O_LOGF(a[i]); break;
        case 5: out[i] = O_POWF(a[i], b[i]); break;
        case 6: out[i] = O_ATAN2F(a[i], b[i]); break;
        case 7: out[i] = O_ACOSF(a[i]); break;
        default: out[i] = NAN; break;
        }
    }
}
