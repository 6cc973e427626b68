// bte_shade.cuh -- device shading for the wavefront stages.
//
// The arithmetic of every function follows the reference's shading headers
// (paths relative to the reference project root, cited per function) in the
// same operation order, because per-sample parity is exact: the stage
// kernels, compiled with -fmad=false, IEEE division and square root, and the
// deterministic elementary functions of bte_math.cuh, reproduce the CPU
// checker bit-for-bit.  What differs from the reference is structural, not
// numerical: BSDF data arrive by value from a per-triangle gather, the
// emitter lookup on a hit is an O(1) side table instead of the linear scan of
// rt_emitter_sampling.cuh:132-148 (same first-match result), texture fetches
// are a software bilinear filter over global memory (the documented hardware
// formula, 8-bit fractional weights), and env-map sampling can use FP64-built
// alias tables in place of the FP32 CDF binary searches.
// Two reference choices are pinned here as documented deviations: rsqrtf in
// normalize3 (rt_cuda_math.cuh:53) is evaluated as 1/sqrtf, and M_PI in
// rt_env_map.cuh:26-28 is the float literal.
#pragma once

#include "bte_math.cuh"
#include "bte_types.cuh"

namespace bte {

// ---------------------------------------------------------------- constants
constexpr float kEps = 1e-4f;                               // rt_constants.cuh:19
constexpr float kPiF = 3.14159265358979323846f;             // rt_bsdf.cuh:11
constexpr float kInvPiF = 1.0f / kPiF;                      // rt_bsdf.cuh:12
constexpr float kAzimuth = 1.0f / (2.0f * kPiF);            // rt_bsdf_microfacet.cuh:11

// ---------------------------------------------------------------- vectors (rt_cuda_math.cuh:8-124)
BTE_DI V3 v3(float x, float y, float z) { return V3{x, y, z}; }
BTE_DI V3 sub3(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
BTE_DI V3 add3(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
BTE_DI V3 mul3(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
BTE_DI V3 mul3(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
BTE_DI V3 div3(V3 a, float s)
{
    if (s == 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const float inv = 1.0f / s;
    return v3(a.x * inv, a.y * inv, a.z * inv);
}
BTE_DI float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
BTE_DI V3 cross3(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
BTE_DI V3 normalize3(V3 v)
{
    const float len2 = dot3(v, v);
    if (len2 <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const float invLen = 1.0f / sqrtf(len2);
    return mul3(v, invLen);
}
BTE_DI float length3(V3 v) { return sqrtf(fmaxf(0.0f, dot3(v, v))); }
BTE_DI float distance3(V3 a, V3 b) { return length3(sub3(a, b)); }
BTE_DI float maxCoeff3(V3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }

struct Frame { V3 t, b, n; };
BTE_DI Frame makeFrame(V3 normal)
{
    Frame f;
    f.n = normalize3(normal);
    const V3 a = (fabsf(f.n.z) < 0.999f) ? v3(0.0f, 0.0f, 1.0f) : v3(1.0f, 0.0f, 0.0f);
    f.t = normalize3(cross3(a, f.n));
    f.b = cross3(f.n, f.t);
    return f;
}
BTE_DI V3 toLocal(const Frame& f, V3 v) { return v3(dot3(v, f.t), dot3(v, f.b), dot3(v, f.n)); }
BTE_DI V3 toWorld(const Frame& f, V3 v) { return add3(add3(mul3(f.t, v.x), mul3(f.b, v.y)), mul3(f.n, v.z)); }

// ---------------------------------------------------------------- RNG (rt_rng.cuh:8-52)
BTE_DI uint32_t hashUint(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
BTE_DI uint32_t rngSeed(uint32_t pixel, uint32_t sampleIndex)
{
    const uint32_t s = hashUint(pixel ^ (sampleIndex * 0x9e3779b9u));
    return s ? s : 1u;
}
BTE_DI float rngNext(uint32_t& s)
{
    uint32_t x = s;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    s = x;
    return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
}

// ---------------------------------------------------------------- texture filter
// Linear filtering with normalized coordinates as documented for tex2D:
// x_B = x*W - 0.5, i = floor(x_B), alpha = frac(x_B) held in 9-bit fixed
// point with 8 fractional bits; wrap / clamp applied to the texel indices.
BTE_DI float texWeight(float frac) { return floorf(frac * 256.0f + 0.5f) * (1.0f / 256.0f); }
BTE_DI int wrapI(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
BTE_DI int clampI(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

BTE_DI float4 texFloat4(const float4* __restrict__ tex, int w, int h, bool wrapV, float u, float v)
{
    float x = u - floorf(u);
    float y = wrapV ? (v - floorf(v)) : fminf(fmaxf(v, 0.0f), 1.0f);
    const float xb = x * static_cast<float>(w) - 0.5f;
    const float yb = y * static_cast<float>(h) - 0.5f;
    const float fx0 = floorf(xb), fy0 = floorf(yb);
    const float a = texWeight(xb - fx0);
    const float b = texWeight(yb - fy0);
    const int ix = static_cast<int>(fx0), iy = static_cast<int>(fy0);
    const int x0 = wrapI(ix, w), x1 = wrapI(ix + 1, w);
    const int y0 = wrapV ? wrapI(iy, h) : clampI(iy, h);
    const int y1 = wrapV ? wrapI(iy + 1, h) : clampI(iy + 1, h);
    const float4 t00 = __ldg(tex + static_cast<size_t>(y0) * w + x0);
    const float4 t10 = __ldg(tex + static_cast<size_t>(y0) * w + x1);
    const float4 t01 = __ldg(tex + static_cast<size_t>(y1) * w + x0);
    const float4 t11 = __ldg(tex + static_cast<size_t>(y1) * w + x1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    float4 r;
    r.x = ((w00 * t00.x + w10 * t10.x) + w01 * t01.x) + w11 * t11.x;
    r.y = ((w00 * t00.y + w10 * t10.y) + w01 * t01.y) + w11 * t11.y;
    r.z = ((w00 * t00.z + w10 * t10.z) + w01 * t01.z) + w11 * t11.z;
    r.w = ((w00 * t00.w + w10 * t10.w) + w01 * t01.w) + w11 * t11.w;
    return r;
}

BTE_DI float4 texRGBA8(const uchar4* __restrict__ tex, int w, int h, float u, float v)
{
    const float x = u - floorf(u), y = v - floorf(v);
    const float xb = x * static_cast<float>(w) - 0.5f;
    const float yb = y * static_cast<float>(h) - 0.5f;
    const float fx0 = floorf(xb), fy0 = floorf(yb);
    const float a = texWeight(xb - fx0);
    const float b = texWeight(yb - fy0);
    const int ix = static_cast<int>(fx0), iy = static_cast<int>(fy0);
    const int x0 = wrapI(ix, w), x1 = wrapI(ix + 1, w);
    const int y0 = wrapI(iy, h), y1 = wrapI(iy + 1, h);
    const uchar4 t00 = tex[static_cast<size_t>(y0) * w + x0];
    const uchar4 t10 = tex[static_cast<size_t>(y0) * w + x1];
    const uchar4 t01 = tex[static_cast<size_t>(y1) * w + x0];
    const uchar4 t11 = tex[static_cast<size_t>(y1) * w + x1];
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    const float k = 1.0f / 255.0f;
    auto ch = [&](unsigned char c00, unsigned char c10, unsigned char c01, unsigned char c11) {
        return ((w00 * (static_cast<float>(c00) * k) + w10 * (static_cast<float>(c10) * k)) +
                w01 * (static_cast<float>(c01) * k)) + w11 * (static_cast<float>(c11) * k);
    };
    return make_float4(ch(t00.x, t10.x, t01.x, t11.x), ch(t00.y, t10.y, t01.y, t11.y),
                       ch(t00.z, t10.z, t01.z, t11.z), ch(t00.w, t10.w, t01.w, t11.w));
}

// ---------------------------------------------------------------- BSDFs
struct BRec { V3 wi, wo; int measure; float eta, rndExtra; };   // rt_bsdf.cuh:19-25
constexpr int kSolid = 1;
BTE_DI BRec brec0() { BRec r; r.wi = v3(0, 0, 0); r.wo = v3(0, 0, 0); r.measure = 0; r.eta = 0.0f; r.rndExtra = 0.0f; return r; }

struct Bsdf { int type; float4 p0, p1, p2, p3; };

// rt_bsdf_diffuse.cuh:15-24
BTE_DI V3 sqCosHemi(float u1, float u2)
{
    const float r = sqrtf(fmaxf(u1, 0.0f));
    const float phi = 2.0f * kPiF * u2;
    float sp, cp;
    m::sincosf_(phi, sp, cp);
    return v3(r * cp, r * sp, sqrtf(fmaxf(0.0f, 1.0f - u1)));
}
// rt_bsdf_diffuse.cuh:27-62
BTE_DI V3 evalDiffuse(const Bsdf& b, const BRec& r)
{
    if (r.measure != kSolid || r.wi.z <= 0.0f || r.wo.z <= 0.0f) return v3(0, 0, 0);
    return mul3(v3(b.p0.x, b.p0.y, b.p0.z), kInvPiF);
}
BTE_DI float pdfDiffuse(const BRec& r)
{
    if (r.measure != kSolid || r.wi.z <= 0.0f || r.wo.z <= 0.0f) return 0.0f;
    return kInvPiF * r.wo.z;
}
BTE_DI V3 sampleDiffuse(const Bsdf& b, BRec& r, float u1, float u2)
{
    if (r.wi.z <= 0.0f) return v3(0, 0, 0);
    r.measure = kSolid;
    r.wo = sqCosHemi(u1, u2);
    r.eta = 1.0f;
    return v3(b.p0.x, b.p0.y, b.p0.z);
}
// rt_bsdf_mirror.cuh:28-33
BTE_DI V3 sampleMirror(const Bsdf& b, BRec& r)
{
    r.wo = v3(-r.wi.x, -r.wi.y, r.wi.z);
    r.eta = 1.0f;
    r.measure = kSolid;
    return v3(b.p0.x, b.p0.y, b.p0.z);
}
// rt_bsdf_dielectric.cuh:13-31
BTE_DI float fresnelDielectric(float cosI, float etaI, float etaT)
{
    if (cosI < 0.0f) { const float t = etaI; etaI = etaT; etaT = t; cosI = -cosI; }
    const float sinT = (etaI / etaT) * sqrtf(fmaxf(0.0f, 1.0f - cosI * cosI));
    if (sinT >= 1.0f) return 1.0f;
    const float cosT = sqrtf(fmaxf(0.0f, 1.0f - sinT * sinT));
    const float Rs = (etaI * cosI - etaT * cosT) / (etaI * cosI + etaT * cosT);
    const float Rp = (etaT * cosI - etaI * cosT) / (etaT * cosI + etaI * cosT);
    return (Rs * Rs + Rp * Rp) * 0.5f;
}
// rt_bsdf_dielectric.cuh:51-103
BTE_DI V3 sampleDielectric(const Bsdf& b, BRec& r, float u1)
{
    r.measure = kSolid;
    V3 res = v3(1.0f, 1.0f, 1.0f);
    float cosI = r.wi.z;
    const float fr = fresnelDielectric(cosI, b.p1.y, b.p1.x);
    if (u1 < fr) {
        r.wo = v3(-r.wi.x, -r.wi.y, r.wi.z);
        r.eta = 1.0f;
    } else {
        float ratio;
        V3 n = v3(0.0f, 0.0f, 1.0f);
        if (cosI > 0) ratio = b.p1.y / b.p1.x;
        else { ratio = b.p1.x / b.p1.y; n = v3(0.0f, 0.0f, -1.0f); }
        cosI = fabsf(cosI);
        const float root = 1.0f - (ratio * ratio) * (1.0f - cosI * cosI);
        const float dia = ratio * cosI - sqrtf(root);
        r.wo = v3(-ratio * r.wi.x + dia * n.x, -ratio * r.wi.y + dia * n.y, -ratio * r.wi.z + dia * n.z);
        r.eta = 1.0f / ratio;
        const float w = ratio * ratio;
        res = v3(w, w, w);
    }
    return res;
}
// rt_bsdf_microfacet.cuh:23-185
BTE_DI float tanThetaMf(V3 w)
{
    const float ct = w.z;
    const float s2 = fmaxf(0.0f, 1.0f - ct * ct);
    const float c2 = ct * ct;
    if (c2 <= 0.0f) return 0.0f;
    return sqrtf(s2 / c2);
}
BTE_DI V3 sqBeckmann(float u1, float u2, float alpha)
{
    const float phi = 2.0f * kPiF * u2;
    const float tan2 = -alpha * alpha * m::logf_(fmaxf(1.0e-6f, 1.0f - u1));
    const float c = 1.0f / sqrtf(1.0f + tan2);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float sp, cp;
    m::sincosf_(phi, sp, cp);
    return v3(s * cp, s * sp, c);
}
BTE_DI float sqBeckmannPdf(V3 mm, float alpha)
{
    if (mm.z <= 0.0f) return 0.0f;
    const float t = tanThetaMf(mm);
    const float a2 = alpha * alpha;
    const float c = mm.z;
    const float c3 = c * c * c;
    return kAzimuth * (2.0f * m::expf_(-1.0f * t * t / a2)) / (a2 * c3);
}
BTE_DI float shadowMaskMf(const Bsdf& b, V3 wv, V3 wh)
{
    const float c = dot3(wv, wh) / wv.z;
    if (c <= 0.0f) return 0.0f;
    const float bb = 1.0f / (b.p1.x * tanThetaMf(wv));
    if (bb < 1.6f) return ((3.535f * bb) + 2.181f * bb * bb) / (1.0f + (2.276f * bb) + 2.577f * bb * bb);
    return 1.0f;
}
BTE_DI V3 evalMicrofacet(const Bsdf& b, const BRec& r)
{
    if (r.measure != kSolid || r.wi.z <= 0.0f || r.wo.z <= 0.0f) return v3(0, 0, 0);
    const float alpha = b.p1.x;
    const V3 diff = v3(b.p0.x * kInvPiF, b.p0.y * kInvPiF, b.p0.z * kInvPiF);
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float tanH = tanThetaMf(wh);
    const float cosH = wh.z;
    const float num = 2.0f * m::expf_(-1.0f * tanH * tanH / (alpha * alpha));
    const float den = alpha * alpha * cosH * cosH * cosH;
    const float D = kAzimuth * num / den;
    const float F = fresnelDielectric(dot3(wh, r.wi), b.p1.z, b.p1.y);
    const float G = shadowMaskMf(b, r.wi, wh) * shadowMaskMf(b, r.wo, wh);
    const float ecf = 4.0f * r.wi.z * cosH * r.wo.z;
    const float spec = b.p1.w * (D * F * G) / ecf;
    return v3(diff.x + spec, diff.y + spec, diff.z + spec);
}
BTE_DI float pdfMicrofacet(const Bsdf& b, const BRec& r)
{
    if (r.measure != kSolid || r.wi.z <= 0.0f || r.wo.z <= 0.0f) return 0.0f;
    const float cosPdf = (r.wo.z <= 0.0f) ? 0.0f : kInvPiF * r.wo.z;
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float bp = sqBeckmannPdf(wh, b.p1.x);
    const float jac = 1.0f / (4.0f * dot3(wh, r.wo));
    return b.p1.w * bp * jac + (1.0f - b.p1.w) * cosPdf;
}
BTE_DI V3 sampleMicrofacet(const Bsdf& b, BRec& r, float u1, float u2)
{
    if (r.wi.z <= 0.0f) return v3(0, 0, 0);
    float sx = u1;
    bool spec;
    if (sx < b.p1.w) { spec = true; sx = sx / b.p1.w; }
    else { spec = false; sx = (sx - b.p1.w) / (1.0f - b.p1.w); }
    r.measure = kSolid;
    r.eta = 1.0f;
    if (spec) {
        const V3 mm = sqBeckmann(sx, u2, b.p1.x);
        r.wo = sub3(mul3(mm, 2.0f * dot3(r.wi, mm)), r.wi);
    } else {
        r.wo = sqCosHemi(sx, u2);
    }
    if (r.wo.z <= 0.0f) return v3(0, 0, 0);
    const float p = pdfMicrofacet(b, r);
    if (p <= 0.0f) return v3(0, 0, 0);
    return mul3(evalMicrofacet(b, r), r.wo.z / p);
}

// ---- Disney: rt_bsdf_disney.cuh:16-892 ----
BTE_DI V3 dBase(const Bsdf& b) { return v3(b.p0.x, b.p0.y, b.p0.z); }
BTE_DI V3 dSqrt3(V3 c) { return v3(sqrtf(fmaxf(0.0f, c.x)), sqrtf(fmaxf(0.0f, c.y)), sqrtf(fmaxf(0.0f, c.z))); }
BTE_DI float dDiffF(float c, float f90) { return 1.0f + ((f90 - 1.0f) * m::pow5f_(1.0f - c)); }
BTE_DI V3 evalDiffuseLobe(const Bsdf& b, const BRec& r)            // :59-104
{
    const float ci = r.wi.z, co = r.wo.z;
    if (ci <= 0.0f || co <= 0.0f) return v3(0, 0, 0);
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float hDotWo = fabsf(dot3(wh, r.wo));
    const float dfN = 0.5f + (2.0f * b.p0.w * hDotWo * hDotWo);
    const float ssN = b.p0.w * hDotWo * hDotWo;
    const V3 cop = div3(dBase(b), kPiF);
    const V3 base = mul3(cop, dDiffF(ci, dfN) * dDiffF(co, dfN) * co);
    const float ssDen = fmaxf(1e-2f, ci + co);
    const V3 ss = mul3(cop, 1.25f * (dDiffF(ci, ssN) * dDiffF(co, ssN) * ((1.0f / ssDen) - 0.5f) + 0.5f) * co);
    return add3(mul3(base, 1.0f - b.p2.z), mul3(ss, b.p2.z));
}
BTE_DI float pdfCosLobe(const BRec& r)                              // :107-124, :712-730
{
    if (r.measure != kSolid || r.wi.z <= 0 || r.wo.z <= 0) return 0.0f;
    return kInvPiF * r.wo.z;
}
BTE_DI float schlickF0(float eta) { const float n = eta - 1.0f, d = eta + 1.0f; return (n * n) / (d * d); }
BTE_DI V3 fresnelMetal(const Bsdf& b, float hDotWo)                // :157-184
{
    const V3 bc = dBase(b);
    const float lumi = 0.3f * bc.x + 0.6f * bc.y + 0.1f * bc.z;
    V3 tint = v3(1.0f, 1.0f, 1.0f);
    if (lumi > 0) tint = div3(bc, lumi);
    const float st = b.p1.w;
    const V3 sp = v3((1.0f - st) + (st * tint.x), (1.0f - st) + (st * tint.y), (1.0f - st) + (st * tint.z));
    const float coef = b.p1.y * schlickF0(b.p3.z) * (1.0f - b.p1.x);
    const V3 clr = v3((coef * sp.x) + (bc.x * b.p1.x), (coef * sp.y) + (bc.y * b.p1.x), (coef * sp.z) + (bc.z * b.p1.x));
    const float sch = m::pow5f_(1.0f - hDotWo);
    return v3(clr.x + ((1.0f - clr.x) * sch), clr.y + ((1.0f - clr.y) * sch), clr.z + ((1.0f - clr.z) * sch));
}
BTE_DI float ggxD(V3 wh, float ax, float ay)                        // :186-192
{
    const float den = kPiF * ax * ay *
                      m::pow2f_(((wh.x * wh.x) / (ax * ax)) + ((wh.y * wh.y) / (ay * ay)) + (wh.z * wh.z));
    return 1.0f / den;
}
BTE_DI float lambdaG(V3 w, float ax, float ay)                      // :194-204
{
    const float axw = w.x * ax, ayw = w.y * ay;
    const float num = sqrtf(1 + (((axw * axw) + (ayw * ayw)) / fmaxf(1e-8f, (w.z * w.z)))) - 1.0f;
    const float lam = num / 2.0f;
    return 1.0f / (1.0f + lam);
}
BTE_DI void dAlpha(const Bsdf& b, float& ax, float& ay)             // :226-231
{
    const float aspect = sqrtf(1.0f - (0.9f * b.p2.w));
    ax = fmaxf(static_cast<float>(0.0001), (b.p0.w * b.p0.w) / aspect);
    ay = fmaxf(static_cast<float>(0.0001), (b.p0.w * b.p0.w) * aspect);
}
BTE_DI V3 evalMetalLobe(const Bsdf& b, const BRec& r)               // :213-241
{
    const float ci = r.wi.z;
    if (ci <= 0.0f || r.wo.z <= 0.0f) return v3(0, 0, 0);
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float hDotWo = fabsf(dot3(wh, r.wo));
    float ax, ay; dAlpha(b, ax, ay);
    const V3 fm = fresnelMetal(b, hDotWo);
    const float dm = ggxD(wh, ax, ay);
    const float gm = lambdaG(r.wi, ax, ay) * lambdaG(r.wo, ax, ay);
    return div3(mul3(fm, dm * gm), (4 * ci));
}
BTE_DI float pdfMetalLobe(const Bsdf& b, const BRec& r)             // :244-271
{
    const float ci = r.wi.z;
    if (ci <= 0.0f || r.wo.z <= 0.0f) return 0.0f;
    const V3 wh = normalize3(add3(r.wi, r.wo));
    float ax, ay; dAlpha(b, ax, ay);
    const float dm = ggxD(wh, ax, ay);
    const float gm = lambdaG(r.wi, ax, ay);
    const float hDotWi = fabsf(dot3(wh, r.wi));
    const float hDotWo = fabsf(dot3(wh, r.wo));
    return (dm * gm * hDotWi) / (ci * 4.0f * hDotWo);
}
BTE_DI V3 vndf(V3 w, float ax, float ay, float u1, float u2)        // :293-317 and :610-634
{
    const V3 vh = normalize3(v3(ax * w.x, ay * w.y, w.z));
    const float pl = (vh.x * vh.x) + (vh.y * vh.y);
    V3 o1 = v3(1.0f, 0.0f, 0.0f);
    if (pl > 0.0f) o1 = div3(v3(-1.0f * vh.y, vh.x, 0.0f), sqrtf(pl));
    const V3 o2 = cross3(vh, o1);
    const float radius = sqrtf(u1);
    const float phi = 2.0f * kPiF * u2;
    float sphi, cphi;
    m::sincosf_(phi, sphi, cphi);
    const float t1 = radius * cphi;
    float t2 = radius * sphi;
    const float skew = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - skew) * sqrtf(1.0f - (t1 * t1)) + (skew * t2);
    const V3 ph = add3(add3(mul3(o1, t1), mul3(o2, t2)), mul3(vh, sqrtf(fmaxf(0.0f, 1 - (t1 * t1) - (t2 * t2)))));
    return normalize3(v3(ax * ph.x, ay * ph.y, fmaxf(0.0f, ph.z)));
}
BTE_DI V3 sampleMetalLobe(const Bsdf& b, BRec& r, float u1, float u2)   // :274-335
{
    if (r.wi.z <= 0.0f) return v3(0, 0, 0);
    r.measure = kSolid;
    r.eta = 1.0f;
    float ax, ay; dAlpha(b, ax, ay);
    const V3 h = vndf(r.wi, ax, ay, u1, u2);
    r.wo = sub3(mul3(h, 2.0f * dot3(r.wi, h)), r.wi);
    if (r.wo.z <= 0.0f) return v3(0, 0, 0);
    const float hDotWo = fabsf(dot3(h, r.wo));
    return mul3(fresnelMetal(b, hDotWo), lambdaG(r.wo, ax, ay));
}
BTE_DI float clearD(const Bsdf& b, V3 wh)                           // :351-363
{
    const float ir = ((1.0f - b.p3.y) * 0.1f) + (b.p3.y * 0.001f);
    const float ir2 = ir * ir;
    const float num = ir2 - 1.0f;
    const float den = kPiF * m::logf_(ir2) * (1.0f + ((ir2 - 1.0f) * (wh.z * wh.z)));
    return num / den;
}
BTE_DI V3 evalClearLobe(const Bsdf& b, const BRec& r)               // :370-394
{
    const float ci = r.wi.z;
    if (ci <= 0.0f || r.wo.z <= 0.0f) return v3(0, 0, 0);
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float hDotWo = fabsf(dot3(wh, r.wo));
    const float rr = static_cast<float>(0.04);
    const float fc = rr + ((1.0f - rr) * m::pow5f_(1.0f - hDotWo));
    const float dc = clearD(b, wh);
    const float gc = lambdaG(r.wi, 0.25f, 0.25f) * lambdaG(r.wo, 0.25f, 0.25f);
    const float den = 4.0f * ci;
    const float cc = (fc * dc * gc) / den;
    return v3(cc, cc, cc);
}
BTE_DI float pdfClearLobe(const Bsdf& b, const BRec& r)             // :397-414
{
    const float ci = r.wi.z;
    if (ci <= 0.0f || r.wo.z <= 0.0f) return 0.0f;
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float dc = clearD(b, wh);
    const float hDotWo = fabsf(dot3(wh, r.wo));
    return (dc * wh.z) / (4.0f * hDotWo);
}
BTE_DI V3 sampleClearLobe(const Bsdf& b, BRec& r, float u1, float u2)   // :417-450
{
    if (r.wi.z <= 0.0f) return v3(0, 0, 0);
    r.measure = kSolid;
    const float ir = ((1.0f - b.p3.y) * 0.1f) + (b.p3.y * 0.001f);
    const float ir2 = ir * ir;
    const float az = 2.0f * kPiF * u1;
    const float ce2 = (1.0f - m::powf_(ir2, 1.0f - u2)) / (1.0f - ir2);
    const float se = sqrtf(1.0f - ce2);
    const float hz = sqrtf(ce2);
    float saz, caz;
    m::sincosf_(az, saz, caz);
    const float hy = se * saz;
    const float hx = se * caz;
    const V3 wh = normalize3(v3(hx, hy, hz));
    r.wo = sub3(mul3(wh, 2.0f * dot3(r.wi, wh)), r.wi);
    r.eta = 1.0f;
    if (r.wo.z <= 0.0f) return v3(0, 0, 0);
    return div3(evalClearLobe(b, r), pdfClearLobe(b, r));
}
BTE_DI float fresnelGlass(float hi, float ho, float ehi, float eho) // :455-472
{
    hi = fabsf(hi); ho = fabsf(ho); ehi = fabsf(ehi); eho = fabsf(eho);
    const float rs = (hi - eho) / (hi + eho);
    const float rp = (ehi - ho) / (ehi + ho);
    return 0.5f * ((rs * rs) + (rp * rp));
}
BTE_DI V3 glassHalf(const BRec& r, float eta, float inNout)        // :486-498
{
    V3 wh;
    if (inNout > 0.0f) wh = normalize3(add3(r.wi, r.wo));
    else wh = mul3(normalize3(add3(r.wi, mul3(r.wo, eta))), -1.0f);
    if (wh.z < 0.0f) wh = mul3(wh, -1.0f);
    return wh;
}
BTE_DI V3 evalGlassLobe(const Bsdf& b, const BRec& r)               // :475-532
{
    const float ci = r.wi.z, co = r.wo.z;
    float eta = b.p3.z;
    if (ci < 0.0f) eta = 1.0f / eta;
    const float inNout = ci * co;
    const V3 wh = glassHalf(r, eta, inNout);
    const float hDotWi = dot3(wh, r.wi), hDotWo = dot3(wh, r.wo);
    const float ehi = eta * hDotWi, eho = eta * hDotWo;
    const float fg = fresnelGlass(hDotWi, hDotWo, ehi, eho);
    float ax, ay; dAlpha(b, ax, ay);
    const float dg = ggxD(wh, ax, ay);
    const float gg = lambdaG(r.wi, ax, ay) * lambdaG(r.wo, ax, ay);
    if (inNout > 0.0f) {
        const V3 num = mul3(dBase(b), fg * dg * gg);
        const float den = 4.0f * fabsf(ci);
        return div3(num, den);
    }
    const V3 num = mul3(dSqrt3(dBase(b)), (1.0f - fg) * dg * gg * fabsf(hDotWi * hDotWo));
    const float den = fabsf(ci) * fmaxf(m::pow2f_(hDotWi + eho), 1e-4f);
    return div3(num, den);
}
BTE_DI float pdfGlassLobe(const Bsdf& b, const BRec& r)             // :535-588
{
    const float ci = r.wi.z, co = r.wo.z;
    float eta = b.p3.z;
    if (ci < 0.0f) eta = 1.0f / eta;
    const float inNout = ci * co;
    const V3 wh = glassHalf(r, eta, inNout);
    const float hDotWi = dot3(wh, r.wi), hDotWo = dot3(wh, r.wo);
    const float fg = fresnelGlass(hDotWi, hDotWo, eta * hDotWi, eta * hDotWo);
    float ax, ay; dAlpha(b, ax, ay);
    const float dg = ggxD(wh, ax, ay);
    const float gg = lambdaG(r.wi, ax, ay);
    const float common = (dg * gg * fabsf(hDotWi)) / fabsf(ci);
    if (inNout > 0.0f) return (common * fg) / (4.0f * fabsf(hDotWo));
    const float jac = (eta * eta * fabsf(hDotWo)) / fmaxf(m::pow2f_(hDotWi + (eta * hDotWo)), 1e-4f);
    return (1.0f - fg) * common * jac;
}
BTE_DI V3 sampleGlassLobe(const Bsdf& b, BRec& r, float u1, float u2)   // :591-674
{
    const float ci = r.wi.z;
    r.measure = kSolid;
    float ax, ay; dAlpha(b, ax, ay);
    float eta = b.p3.z;
    if (ci < 0.0f) eta = 1.0f / eta;
    const V3 wiU = (ci < 0.0f) ? mul3(r.wi, -1.0f) : r.wi;
    V3 h = vndf(wiU, ax, ay, u1, u2);
    if (ci < 0.0f) h = mul3(h, -1.0f);
    const float hDotWi = dot3(h, r.wi);
    const float sin2T = (1.0f - hDotWi * hDotWi) / (eta * eta);
    const float hDotWt = sqrtf(fmaxf(0.0f, 1.0f - sin2T));
    const float fg = fresnelGlass(hDotWi, hDotWt, eta * hDotWi, eta * hDotWt);
    if (r.rndExtra < fg || sin2T >= 1.0f) {
        r.wo = sub3(mul3(h, 2.0f * dot3(r.wi, h)), r.wi);
        r.eta = 1.0f;
    } else {
        r.wo = sub3(mul3(h, (hDotWi / eta) - hDotWt), div3(r.wi, eta));
        r.wo = normalize3(r.wo);
        r.eta = eta;
    }
    const float pdf = pdfGlassLobe(b, r);
    if (pdf == 0.0f) return v3(0, 0, 0);
    return div3(evalGlassLobe(b, r), pdf);
}
BTE_DI V3 evalSheenLobe(const Bsdf& b, const BRec& r)               // :679-709
{
    const float ci = r.wi.z, co = r.wo.z;
    if (ci <= 0.0f || co <= 0.0f) return v3(0, 0, 0);
    const V3 wh = normalize3(add3(r.wi, r.wo));
    const float hDotWo = fabsf(dot3(wh, r.wo));
    const V3 bc = dBase(b);
    const float lumi = 0.3f * bc.x + 0.6f * bc.y + 0.1f * bc.z;
    V3 tint = v3(1.0f, 1.0f, 1.0f);
    if (lumi > 0) tint = div3(bc, lumi);
    const float st = b.p2.y;
    const V3 sh = v3((1.0f - st) + (st * tint.x), (1.0f - st) + (st * tint.y), (1.0f - st) + (st * tint.z));
    return mul3(sh, m::pow5f_(1.0f - hDotWo) * co);
}
BTE_DI V3 evalDisney(const Bsdf& b, const BRec& r)                  // :758-787
{
    if (r.wi.z <= 0.0f) {
        if (b.p1.z <= 0.0f) return v3(0, 0, 0);
        return evalGlassLobe(b, r);
    }
    const float minMetal = (1.0f - b.p1.x);
    const float minST = (1.0f - b.p1.z);
    const V3 fd = mul3(evalDiffuseLobe(b, r), minMetal * minST);
    const V3 fs = mul3(evalSheenLobe(b, r), minMetal * b.p2.x);
    const V3 fm = mul3(evalMetalLobe(b, r), (1.0f - (b.p1.z * minMetal)));
    const V3 fc = mul3(evalClearLobe(b, r), 0.25f * b.p3.x);
    const V3 fg = mul3(evalGlassLobe(b, r), minMetal * b.p1.z);
    return add3(add3(add3(add3(fd, fm), fg), fc), fs);
}
BTE_DI float pdfDisney(const Bsdf& b, const BRec& r)                // :790-820
{
    const float minMetal = (1.0f - b.p1.x);
    const float minST = (1.0f - b.p1.z);
    const float dW = minMetal * minST;
    const float mW = 1.0f - (b.p1.z * minMetal);
    const float gW = minMetal * b.p1.z;
    const float cW = 0.25f * b.p3.x;
    const float wSum = dW + gW + mW + cW;
    if (r.wi.z <= 0) {
        if (b.p1.z <= 0.0f) return 0.0f;
        return pdfGlassLobe(b, r);
    }
    const float pD = pdfCosLobe(r);
    const float pM = pdfMetalLobe(b, r);
    const float pG = pdfGlassLobe(b, r);
    const float pC = pdfClearLobe(b, r);
    return (dW * pD + gW * pG + mW * pM + cW * pC) / wSum;
}
BTE_DI V3 sampleDisney(const Bsdf& b, BRec& r, float u1, float u2)  // :823-892
{
    if (r.wi.z <= 0.0f) {
        if (b.p1.z <= 0.0f) return v3(0, 0, 0);
        sampleGlassLobe(b, r, u1, u2);
    } else {
        const float minMetal = (1.0f - b.p1.x);
        const float dW = minMetal * (1.0f - b.p1.z);
        const float sW = minMetal * b.p1.z;
        const float mW = 1.0f - (b.p1.z * minMetal);
        const float cW = 0.25f * b.p3.x;
        const float wSum = dW + sW + mW + cW;
        const float rc = r.rndExtra;
        const float dF = dW / wSum, sF = sW / wSum, mF = mW / wSum;
        if (rc < dF) {
            if (r.wi.z > 0) {   // sampleDiffuseLobe :127-146 (its return value is discarded)
                r.measure = kSolid;
                r.wo = sqCosHemi(u1, u2);
                r.eta = 1.0f;
            }
        } else if (rc < dF + sF) {
            r.rndExtra = (sF > 0.0f) ? (rc - dF) / sF : 0.0f;
            sampleGlassLobe(b, r, u1, u2);
        } else if (rc < dF + sF + mF) {
            sampleMetalLobe(b, r, u1, u2);
        } else {
            sampleClearLobe(b, r, u1, u2);
        }
    }
    const float pdf = pdfDisney(b, r);
    if (pdf < 1e-7f) return v3(0, 0, 0);
    return div3(evalDisney(b, r), pdf);
}

// dispatch, rt_bsdf.cuh:42-84.  The product build (BTE_FAST_MATH) inlines the three: material-sorted shading gives
// a warp one BSDF, and inlining drops the by-reference argument records in local memory (1080p bench frame
// 7.76 -> 7.69 ms, shade 2.29 -> 2.25 ms).  The parity build keeps one out-of-line copy of each beside its
// out-of-line double-evaluated math functions.
#if defined(BTE_FAST_MATH) || defined(BTE_BSDF_INLINE)
#define BTE_BSDF_FN __device__ __forceinline__
#else
#define BTE_BSDF_FN __device__ __noinline__
#endif
BTE_BSDF_FN V3 bsdfEval(const Bsdf& b, const BRec& r)
{
    switch (b.type) {
    case BSDF_Diffuse: return evalDiffuse(b, r);
    case BSDF_Microfacet: return evalMicrofacet(b, r);
    case BSDF_Disney: return evalDisney(b, r);
    default: return v3(0, 0, 0);
    }
}
BTE_BSDF_FN float bsdfPdf(const Bsdf& b, const BRec& r)
{
    switch (b.type) {
    case BSDF_Diffuse: return pdfDiffuse(r);
    case BSDF_Microfacet: return pdfMicrofacet(b, r);
    case BSDF_Disney: return pdfDisney(b, r);
    default: return 0.0f;
    }
}
BTE_BSDF_FN V3 bsdfSample(const Bsdf& b, BRec& r, float u1, float u2)
{
    switch (b.type) {
    case BSDF_Diffuse: return sampleDiffuse(b, r, u1, u2);
    case BSDF_Dielectric: return sampleDielectric(b, r, u1);
    case BSDF_Mirror: return sampleMirror(b, r);
    case BSDF_Microfacet: return sampleMicrofacet(b, r, u1, u2);
    case BSDF_Disney: return sampleDisney(b, r, u1, u2);
    default: return v3(0, 0, 0);
    }
}
BTE_DI bool bsdfIsDiffuseClass(int type) { return type == BSDF_Diffuse || type == BSDF_Microfacet || type == BSDF_Disney; }

// rt_material.cuh:15-59
BTE_DI Bsdf loadBsdf(const DevScene& s, int tri, float u, float v)
{
    const BsdfData& g = s.bsdfs[__ldg(s.triBsdfIds + tri)];
    Bsdf b;
    b.type = g.type;
    b.p0 = make_float4(g.p0.x, g.p0.y, g.p0.z, g.p0.w);
    b.p1 = make_float4(g.p1.x, g.p1.y, g.p1.z, g.p1.w);
    b.p2 = make_float4(g.p2.x, g.p2.y, g.p2.z, g.p2.w);
    b.p3 = make_float4(g.p3.x, g.p3.y, g.p3.z, g.p3.w);
    if (s.texTable != nullptr && s.triMaterialIds != nullptr) {
        const int mi = s.triMaterialIds[tri];
        if (mi >= 0 && mi < s.textureCount) {
            const TexRef t = s.texTable[mi];
            if (t.pixels != nullptr) {
                const float4 c = texRGBA8(t.pixels, t.w, t.h, u, v);
                b.p0.x = c.x; b.p0.y = c.y; b.p0.z = c.z;
                if (b.type == BSDF_Microfacet) b.p1.w = 1.0f - fmaxf(b.p0.x, fmaxf(b.p0.y, b.p0.z));
            }
            if (s.texTableMr != nullptr) {
                const TexRef mr = s.texTableMr[mi];
                if (mr.pixels != nullptr && b.type == BSDF_Disney) {
                    const float4 c = texRGBA8(mr.pixels, mr.w, mr.h, u, v);
                    b.p0.w *= c.y;
                    b.p1.x *= c.z;
                }
            }
        }
    }
    return b;
}

// ---------------------------------------------------------------- environment map (rt_env_map.cuh:36-199)
constexpr float kMPI = 3.14159265358979323846f;
BTE_DI float2 dirToEquirect(V3 d, float rot)
{
    float phi = m::atan2f_(d.z, d.x) + rot;
    const float theta = m::acosf_(fminf(fmaxf(d.y, -1.0f), 1.0f));
    phi = fmodf(phi + kMPI, 2.0f * kMPI);
    if (phi < 0.0f) phi += 2.0f * kMPI;
    phi -= kMPI;
    return make_float2((phi + kMPI) / (2.0f * kMPI), theta / kMPI);
}
BTE_DI V3 equirectToDir(float u, float v, float rot)
{
    const float phi = u * 2.0f * kMPI - kMPI - rot;
    const float theta = v * kMPI;
    float st, ct, sp, cp;
    m::sincosf_(theta, st, ct);
    m::sincosf_(phi, sp, cp);
    return normalize3(v3(st * cp, ct, st * sp));
}
BTE_DI V3 envTex(const DevEnv& e, float u, float v)
{
    const float4 t = texFloat4(e.texels, e.w, e.h, false, u, v);
    return v3(t.x * e.intensity, t.y * e.intensity, t.z * e.intensity);
}
BTE_DI V3 envEval(const DevEnv& e, V3 dir)
{
    const float2 uv = dirToEquirect(dir, e.rotation);
    return envTex(e, uv.x, uv.y);
}
BTE_DI int cdfSearch(const float* __restrict__ cdf, int count, float x)
{
    int lo = 0, hi = count;
    while (lo + 1 < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}
BTE_DI float envSolidAngle(const DevEnv& e, float pPix, float v)
{
    const float theta = v * kMPI;
    const float st = fmaxf(m::sinf_(theta), 1e-6f);
    return (pPix * static_cast<float>(e.w) * static_cast<float>(e.h)) / (2.0f * kMPI * kMPI * st);
}
BTE_DI float envPdf(const DevEnv& e, V3 dir)
{
    if (e.totalPower <= 0.0f) return 0.0f;
    const float2 uv = dirToEquirect(dir, e.rotation);
    const float fx = uv.x * static_cast<float>(e.w);
    const float fy = uv.y * static_cast<float>(e.h);
    const int ix = min(max(static_cast<int>(fx), 0), e.w - 1);
    const int iy = min(max(static_cast<int>(fy), 0), e.h - 1);
    if (e.sampling == BTE_ENV_SAMPLING_ALIAS) {
        const float p = __ldg(e.pixelPdf + static_cast<size_t>(iy) * e.w + ix);
        if (p <= 0.0f) return 0.0f;
        return envSolidAngle(e, p, uv.y);
    }
    const float msum = __ldg(e.marginal + e.h);
    const float rw = __ldg(e.marginal + iy + 1) - __ldg(e.marginal + iy);
    if (msum <= 0.0f || rw <= 0.0f) return 0.0f;
    const float pRow = rw / msum;
    const float* row = e.conditional + static_cast<size_t>(iy) * (e.w + 1);
    const float rsum = __ldg(row + e.w);
    const float cw = __ldg(row + ix + 1) - __ldg(row + ix);
    if (rsum <= 0.0f || cw <= 0.0f) return 0.0f;
    const float pCol = cw / rsum;
    const float theta = uv.y * kMPI;
    const float st = fmaxf(m::sinf_(theta), 1e-6f);
    return (pRow * pCol * static_cast<float>(e.w) * static_cast<float>(e.h)) / (2.0f * kMPI * kMPI * st);
}
struct EnvSample { V3 dir; float pdf; V3 rad; };
BTE_DI int aliasPick(const float* __restrict__ prob, const int* __restrict__ alias, int n, float u, float& frac)
{
    const float x = u * static_cast<float>(n);
    int i = static_cast<int>(x);
    if (i > n - 1) i = n - 1;
    const float f = x - static_cast<float>(i);
    const float p = __ldg(prob + i);
    if (f < p) { frac = f / p; return i; }
    frac = (f - p) / (1.0f - p);
    return __ldg(alias + i);
}
BTE_DI EnvSample envSample(const DevEnv& e, float u0, float u1)
{
    EnvSample r;
    r.dir = v3(0.0f, 1.0f, 0.0f); r.pdf = 0.0f; r.rad = v3(0, 0, 0);
    if (e.totalPower <= 0.0f) return r;
    if (e.sampling == BTE_ENV_SAMPLING_ALIAS) {
        float fr, fc;
        const int row = aliasPick(e.rowProb, e.rowAlias, e.h, u0, fr);
        const int col = aliasPick(e.colProb + static_cast<size_t>(row) * e.w, e.colAlias + static_cast<size_t>(row) * e.w,
                                  e.w, u1, fc);
        if (fr >= 1.0f) fr = 0x1.fffffep-1f;
        if (fc >= 1.0f) fc = 0x1.fffffep-1f;
        const float u = (static_cast<float>(col) + fc) / static_cast<float>(e.w);
        const float v = (static_cast<float>(row) + fr) / static_cast<float>(e.h);
        r.dir = equirectToDir(u, v, e.rotation);
        r.rad = envTex(e, u, v);
        const float p = __ldg(e.pixelPdf + static_cast<size_t>(row) * e.w + col);
        r.pdf = (p > 0.0f) ? envSolidAngle(e, p, v) : 0.0f;
        return r;
    }
    const float msum = __ldg(e.marginal + e.h);
    if (msum <= 0.0f) return r;
    const float xr = u0 * msum;
    const int row = cdfSearch(e.marginal, e.h, xr);
    const float c0r = __ldg(e.marginal + row), c1r = __ldg(e.marginal + row + 1);
    const float dRow = c1r - c0r;
    const float fracRow = (dRow > 0.0f) ? (xr - c0r) / dRow : 0.0f;
    const float* rc = e.conditional + static_cast<size_t>(row) * (e.w + 1);
    const float rsum = __ldg(rc + e.w);
    if (rsum <= 0.0f) return r;
    const float xc = u1 * rsum;
    const int col = cdfSearch(rc, e.w, xc);
    const float c0c = __ldg(rc + col), c1c = __ldg(rc + col + 1);
    const float dCol = c1c - c0c;
    const float fracCol = (dCol > 0.0f) ? (xc - c0c) / dCol : 0.0f;
    const float u = (static_cast<float>(col) + fracCol) / static_cast<float>(e.w);
    const float v = (static_cast<float>(row) + fracRow) / static_cast<float>(e.h);
    r.dir = equirectToDir(u, v, e.rotation);
    r.rad = envTex(e, u, v);
    const float pRow = dRow / msum, pCol = dCol / rsum;
    const float theta = v * kMPI;
    const float st = fmaxf(m::sinf_(theta), 1e-6f);
    r.pdf = (pRow * pCol * static_cast<float>(e.w) * static_cast<float>(e.h)) / (2.0f * kMPI * kMPI * st);
    return r;
}

// ---------------------------------------------------------------- emitters (rt_emitter_sampling.cuh:138-329)
struct EQ { V3 origin, hitPoint, hitNormal; float pdf, emitterPdf; V3 dirToLight; };
BTE_DI EQ eq0() { EQ q; q.origin = q.hitPoint = q.hitNormal = q.dirToLight = v3(0, 0, 0); q.pdf = q.emitterPdf = 0.0f; return q; }

BTE_DI int sampleCdfReuse(const float* __restrict__ cdf, int count, float& u, float& outPdf)
{
    const float sum = __ldg(cdf + count);
    if (sum <= 0.0f || count <= 0) { outPdf = 0.0f; u = 0.0f; return 0; }
    const float x = u * sum;
    int lo = 0, hi = count;
    while (lo + 1 < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= x) lo = mid;
        else hi = mid;
    }
    const float c0 = __ldg(cdf + lo), c1 = __ldg(cdf + lo + 1);
    const float den = c1 - c0;
    if (den <= 0.0f) { u = 0.0f; outPdf = 0.0f; return lo; }
    u = (x - c0) / den;
    outPdf = den / sum;
    return lo;
}
BTE_DI V3 checkRadiance(V3 rad, const EQ& q)
{
    const V3 neg = v3(-q.dirToLight.x, -q.dirToLight.y, -q.dirToLight.z);
    if (dot3(q.hitNormal, neg) <= 0.0f) return v3(0, 0, 0);
    return rad;
}
BTE_DI float sceneEmitterPdf(const DevScene& s, int e)
{
    if (e < 0 || s.emitterCount <= 0 || !s.sceneEmitterCdf) return 0.0f;
    const float sum = s.sceneEmitterCdf[s.emitterCount];
    if (sum <= 0.0f) return 0.0f;
    return (s.sceneEmitterCdf[e + 1] - s.sceneEmitterCdf[e]) / sum;
}
BTE_DI V3 sampleGenerator(const DevScene& s, EQ& q, float u0, float u1)
{
    q.emitterPdf = 0.0f;
    if (s.emitterCount <= 0) return v3(0, 0, 0);
    float epdf = 0.0f;
    const int e = sampleCdfReuse(s.sceneEmitterCdf, s.emitterCount, u0, epdf);
    const EmitterData E = s.emitters[e];
    V3 pos = v3(0, 0, 0), nrm = v3(0, 0, 0);
    float mpdf = 0.0f;
    if (E.triCount > 0) {
        const float* tcdf = s.emitterTriCdf + E.cdfOffset;
        float tp = 0.0f;
        const int li = sampleCdfReuse(tcdf, E.triCount, u0, tp);
        const int ti = __ldg(s.emitterTriIndices + E.triIndexOffset + li);
        const TriangleData& T = s.tris[ti];
        const V3 a = v3(T.v0.x, T.v0.y, T.v0.z), b = v3(T.v1.x, T.v1.y, T.v1.z), c = v3(T.v2.x, T.v2.y, T.v2.z);
        const float root = sqrtf(fmaxf(0.0f, 1.0f - u0));
        const float al = 1.0f - root;
        const float be = u1 * root;
        const float ga = 1.0f - al - be;
        pos = add3(add3(mul3(a, al), mul3(b, be)), mul3(c, ga));
        nrm = normalize3(cross3(sub3(b, a), sub3(c, a)));
        const float area = __ldg(tcdf + E.triCount);
        if (area > 0.0f) mpdf = 1.0f / area;
    }
    q.hitPoint = pos;
    q.hitNormal = nrm;
    q.pdf = mpdf;
    q.dirToLight = normalize3(sub3(q.hitPoint, q.origin));
    q.emitterPdf = epdf;
    return checkRadiance(v3(E.radiance.x, E.radiance.y, E.radiance.z), q);
}

// ---------------------------------------------------------------- path state and lighting
struct PathReg {
    V3 o, d, tp, L;
    float eta, brdfPdf;
    int bounce;
    bool specular;
};
struct HitReg { V3 p, n; float u, v; int tri; };
struct ShadowRec { V3 d; float tmax; V3 c; };

// rt_direct_lighting.cuh:36-49
BTE_DI float areaToSolid(float pA, const EQ& q)
{
    const V3 diff = sub3(q.hitPoint, q.origin);
    const float d2 = dot3(diff, diff);
    const V3 neg = v3(-q.dirToLight.x, -q.dirToLight.y, -q.dirToLight.z);
    const float den = fmaxf(fabsf(dot3(q.hitNormal, neg)), 1e-3f);
    return pA * d2 / den;
}
// :60-99 (emitter lookup through the tri -> emitter side table)
BTE_DI void accumulateEmitterHit(const DevScene& s, PathReg& p, const HitReg& h)
{
    const Float3 r0 = s.emission ? s.emission[h.tri] : Float3{0.0f, 0.0f, 0.0f};
    EQ q = eq0();
    q.origin = p.o; q.hitPoint = h.p; q.hitNormal = h.n; q.dirToLight = p.d;
    float w = 1.0f;
    if (!p.specular) {
        const int e = (s.emitterCount > 0 && s.triEmitter) ? __ldg(s.triEmitter + h.tri) : -1;
        if (e >= 0) {
            const float areaSum = s.emitters[e].areaSum;
            const float ap = (areaSum <= 0.0f) ? 0.0f : 1.0f / areaSum;
            const float pA = ap * sceneEmitterPdf(s, e);
            const float pS = areaToSolid(pA, q);
            const float den = p.brdfPdf + pS;
            if (den <= 0.0f) w = 0.0f;
            else w = p.brdfPdf / den;
        }
    }
    const V3 rad = checkRadiance(v3(r0.x, r0.y, r0.z), q);
    p.L = add3(p.L, mul3(mul3(rad, p.tp), w));
}
// :107-164
BTE_DI bool prepareArea(const DevScene& s, const PathReg& p, uint32_t& rng, const HitReg& h, const Bsdf& b,
                        const V3& wiLocal, const Frame& fr, ShadowRec& sr)
{
    const float ul0 = rngNext(rng);
    const float ul1 = rngNext(rng);
    EQ q = eq0();
    q.origin = h.p;
    const V3 le = sampleGenerator(s, q, ul0, ul1);
    if ((le.x <= 0.0f && le.y <= 0.0f && le.z <= 0.0f) || q.emitterPdf <= 0.0f || q.pdf <= 0.0f) return false;
    const float dist = distance3(q.hitPoint, h.p);
    const float geo = fabsf(dot3(h.n, q.dirToLight)) * fabsf(dot3(q.hitNormal, mul3(q.dirToLight, -1.0f))) / (dist * dist);
    BRec r = brec0();
    r.wi = wiLocal;
    r.wo = toLocal(fr, q.dirToLight);
    r.measure = kSolid;
    const V3 f = bsdfEval(b, r);
    const float pA = q.emitterPdf * q.pdf;
    const float pS = areaToSolid(pA, q);
    const float pB = bsdfPdf(b, r);
    const float den = pB + pS;
    if (den <= 0.0f) return false;
    const float lw = pS / den;
    V3 c = mul3(f, le);
    c = mul3(c, lw);
    c = mul3(c, geo);
    c = div3(c, pA);
    sr.d = q.dirToLight;
    sr.tmax = dist - kEps;
    sr.c = mul3(c, p.tp);
    return true;
}
// :175-230
BTE_DI bool prepareSpot(const DevScene& s, const PathReg& p, const HitReg& h, const Bsdf& b, int si,
                        const V3& wiLocal, const Frame& fr, ShadowRec& sr)
{
    const SpotlightData sp = s.spots[si];
    const V3 o2l = sub3(v3(sp.position.x, sp.position.y, sp.position.z), h.p);
    const float sq = dot3(o2l, o2l);
    if (sq < kEps * kEps) return false;
    const float dist = sqrtf(sq);
    const V3 dl = div3(o2l, dist);
    const float lc = dot3(mul3(dl, -1.0f), v3(sp.direction.x, sp.direction.y, sp.direction.z));
    const V3 rad = v3(sp.radiance.x, sp.radiance.y, sp.radiance.z);
    V3 le;
    if (lc <= sp.outerConeCosine) return false;
    else if (lc >= sp.innerConeCosine) le = mul3(rad, sp.intensity / sq);
    else {
        const float fo = (lc - sp.outerConeCosine) / (sp.innerConeCosine - sp.outerConeCosine);
        const float sm = (fo * fo) * (3.0f - (2.0f * fo));
        le = mul3(rad, (sp.intensity * sm) / sq);
    }
    BRec r = brec0();
    r.wi = wiLocal;
    r.wo = toLocal(fr, dl);
    r.measure = kSolid;
    const V3 f = bsdfEval(b, r);
    const float cs = fabsf(dot3(h.n, dl));
    sr.d = dl;
    sr.tmax = dist - kEps;
    sr.c = mul3(mul3(mul3(f, le), cs), p.tp);
    return true;
}
// :237-259
BTE_DI void accumulateEnvHit(const DevScene& s, PathReg& p)
{
    if (!s.hasEnv) return;
    const V3 er = envEval(s.env, p.d);
    float w = 1.0f;
    if (!p.specular) {
        const float ep = envPdf(s.env, p.d);
        const float sum = p.brdfPdf + ep;
        if (sum > 0.0f) w = p.brdfPdf / sum;
        else w = 0.0f;
    }
    p.L = add3(p.L, mul3(mul3(er, p.tp), w));
}
// :267-315
BTE_DI bool prepareEnv(const DevScene& s, const PathReg& p, uint32_t& rng, const HitReg& h, const Bsdf& b,
                       const V3& wiLocal, const Frame& fr, ShadowRec& sr)
{
    if (!s.hasEnv) return false;
    const float u0 = rngNext(rng);
    const float u1 = rngNext(rng);
    const EnvSample es = envSample(s.env, u0, u1);
    if (es.pdf <= 0.0f) return false;
    if (es.rad.x <= 0.0f && es.rad.y <= 0.0f && es.rad.z <= 0.0f) return false;
    const float ca = dot3(h.n, es.dir);
    if (ca <= 0.0f) return false;
    BRec r = brec0();
    r.wi = wiLocal;
    r.wo = toLocal(fr, es.dir);
    r.measure = kSolid;
    const V3 f = bsdfEval(b, r);
    const float bp = bsdfPdf(b, r);
    const float sum = bp + es.pdf;
    if (sum <= 0.0f) return false;
    const float lw = es.pdf / sum;
    V3 c = mul3(f, es.rad);
    c = mul3(c, ca);
    c = div3(c, es.pdf);
    c = mul3(c, lw);
    sr.d = es.dir;
    sr.tmax = 1e30f - kEps;
    sr.c = mul3(c, p.tp);
    return true;
}
// rt_path_integrator.cuh:25-47
BTE_DI void scatter(PathReg& p, uint32_t& rng, const HitReg& h, const Bsdf& b, const V3& wiLocal, const Frame& fr)
{
    BRec r = brec0();
    r.wi = wiLocal;
    r.rndExtra = rngNext(rng);
    const float u0 = rngNext(rng);
    const float u1 = rngNext(rng);
    const V3 sw = bsdfSample(b, r, u0, u1);
    p.brdfPdf = bsdfPdf(b, r);
    const V3 bd = normalize3(toWorld(fr, r.wo));
    p.o = add3(h.p, mul3(bd, kEps));
    p.d = bd;
    p.tp = mul3(p.tp, sw);
    p.eta *= r.eta;
}
// :54-65
BTE_DI bool roulette(PathReg& p, uint32_t& rng, int rrStart)
{
    if (p.bounce > rrStart) {
        const float cp = fminf(maxCoeff3(p.tp) * p.eta * p.eta, 0.99f);
        if (rngNext(rng) >= cp) return false;
        p.tp = div3(p.tp, cp);
    }
    return true;
}

// rt_camera.cuh:15-37 (tan(fov/2) evaluated once per frame with the same tanf_)
BTE_DI void primaryRay(int px, int py, int w, int h, const CameraData& c, float tanHalf, float jx, float jy, V3& o, V3& d)
{
    const float fx = (static_cast<float>(px) + 0.5f + jx) / static_cast<float>(w);
    const float fy = (static_cast<float>(py) + 0.5f + jy) / static_cast<float>(h);
    const float ndcX = 2.0f * fx - 1.0f;
    const float ndcY = 2.0f * fy - 1.0f;
    const float sx = ndcX * c.aspect * tanHalf;
    const float sy = ndcY * tanHalf;
    const V3 fwd = v3(c.forward.x, c.forward.y, c.forward.z);
    const V3 rt = v3(c.right.x, c.right.y, c.right.z);
    const V3 up = v3(c.up.x, c.up.y, c.up.z);
    o = v3(c.origin.x, c.origin.y, c.origin.z);
    d = normalize3(add3(fwd, add3(mul3(rt, sx), mul3(up, sy))));
}

// rt_path_integrator.cuh:93-105
BTE_DI uint32_t packGamma(float r, float g, float b)
{
    const float dr = m::powf_(fmaxf(0.0f, fminf(r, 1.0f)), 1.0f / 2.2f);
    const float dg = m::powf_(fmaxf(0.0f, fminf(g, 1.0f)), 1.0f / 2.2f);
    const float db = m::powf_(fmaxf(0.0f, fminf(b, 1.0f)), 1.0f / 2.2f);
    const uint32_t R = static_cast<uint8_t>(dr * 255.0f), G = static_cast<uint8_t>(dg * 255.0f),
                   B = static_cast<uint8_t>(db * 255.0f);
    return (255u << 24) | (B << 16) | (G << 8) | R;
}

}  // namespace bte
