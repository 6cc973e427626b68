/*
 * oracle/ref_harness.cpp -- ORACLE (test infrastructure only).
 *
 * Compiles the reference's own trace-free shading headers (include/rt_*.cuh,
 * include/wavefront/*.cuh, used where they lie under the reference tree) as
 * host C++ through oracle/ref_shim/cuda_runtime.h, and drives them exactly
 * as the reference's per-path loop does:
 *   generate: src/wavefront/ray_generate.cu:49-73
 *   bounce:   src/optix_programs.cu:85-95 calling the body of traceRay,
 *             include/rt_optix_shading.cuh:412-447 (identical in order to the
 *             wavefront shade kernel, src/wavefront/ray_shade.cu:103-183)
 *   closest-hit attributes: src/optix_programs.cu:110-141
 * OptiX is closed and unavailable, so the traversal (closest hit and
 * occlusion in [1e-4, tmax]) is the oracle's watertight CPU traversal
 * (oracle/bte_oracle.c); everything else is the reference's code.
 *
 * Exported entry points mirror oracle/bte_oracle.h with a ref_ prefix, so
 * tests can compare the oracle restatement with the reference bit-for-bit.
 * Built by oracle/Makefile into oracle/_ref/libbteref.so (never committed).
 */
#include <cuda_runtime.h>   // the shim

#include "render_kernel.h"
#include "rt_cuda_math.cuh"
#include "rt_rng.cuh"
#include "rt_camera.cuh"
#include "rt_bsdf.cuh"
#include "rt_emitter_sampling.cuh"
#include "rt_shading_context.cuh"
#include "rt_material.cuh"
#include "rt_env_map.cuh"
#include "rt_direct_lighting.cuh"
#include "rt_path_integrator.cuh"
#include "rt_constants.cuh"
#include "wavefront/wavefront_buffers.h"
#include "wavefront/wavefront_shading.cuh"

#include "bte_oracle.h"

#include <vector>
#include <mutex>
#ifdef _OPENMP
#include <omp.h>
#endif

#define REF_API extern "C" __attribute__((visibility("default")))

static_assert(sizeof(TriangleData) == sizeof(OTri), "TriangleData layout");
static_assert(sizeof(BsdfData) == sizeof(OBsdf), "BsdfData layout");
static_assert(sizeof(EmitterData) == sizeof(OEmitter), "EmitterData layout");
static_assert(sizeof(SpotlightData) == sizeof(OSpot), "SpotlightData layout");
static_assert(sizeof(CameraData) == sizeof(OCamera), "CameraData layout");

// ---------------------------------------------------------------------------
// texture registry behind the shim's tex2D<float4>
// ---------------------------------------------------------------------------
namespace {
struct RefTexture {
    const float* f4 = nullptr;     // float4 texels (env map)
    const uint8_t* rgba8 = nullptr; // RGBA8 texels (material maps)
    int w = 0, h = 0;
    int wrapV = 1;
};
std::vector<RefTexture> g_textures(1);   // handle 0 = "no texture"
std::mutex g_texMutex;

cudaTextureObject_t registerTexture(const RefTexture& t)
{
    std::lock_guard<std::mutex> lk(g_texMutex);
    g_textures.push_back(t);
    return static_cast<cudaTextureObject_t>(g_textures.size() - 1);
}
void resetTextures()
{
    std::lock_guard<std::mutex> lk(g_texMutex);
    g_textures.resize(1);
}
}  // namespace

extern "C" float4 bte_ref_tex2d_float4(cudaTextureObject_t obj, float u, float v)
{
    float out[4] = {0, 0, 0, 0};
    const RefTexture& t = g_textures[static_cast<size_t>(obj)];
    if (t.f4) or_tex_sample_f4(t.f4, t.w, t.h, t.wrapV, u, v, out);
    else if (t.rgba8) or_tex_sample_rgba8(t.rgba8, t.w, t.h, u, v, out);
    return float4{out[0], out[1], out[2], out[3]};
}

// ---------------------------------------------------------------------------
// scene view assembly (what wavefront_host.cu:122-148 packs on the device)
// ---------------------------------------------------------------------------
namespace {
struct RefScene {
    WfSceneView sv{};
    std::vector<cudaTextureObject_t> tex, texMr;
};

void buildRefScene(const OScene* s, RefScene& r)
{
    resetTextures();
    WfSceneView& sv = r.sv;
    sv.triangles = reinterpret_cast<const TriangleData*>(s->triangles);
    sv.triangleCount = s->triangleCount;
    sv.triangleEmitterFlags = s->emitterFlags;
    sv.triangleEmission = reinterpret_cast<const Float3*>(s->emission);
    sv.bsdfs = reinterpret_cast<const BsdfData*>(s->bsdfs);
    sv.bsdfCount = s->bsdfCount;
    sv.triangleBsdfIds = s->triBsdfIds;
    sv.triangleMaterialIds = s->triMaterialIds;
    sv.emitters = reinterpret_cast<const EmitterData*>(s->emitters);
    sv.emitterCount = s->emitterCount;
    sv.emitterTriIndices = s->emitterTriIndices;
    sv.emitterTriCdf = s->emitterTriCdf;
    sv.sceneEmitterCdf = s->sceneEmitterCdf;
    sv.spotlights = reinterpret_cast<const SpotlightData*>(s->spots);
    sv.spotlightCount = s->spotCount;
    sv.texObjects = nullptr;
    sv.texObjectsMr = nullptr;
    sv.textureCount = 0;
    if (s->texPixels && s->textureCount > 0) {
        r.tex.assign(static_cast<size_t>(s->textureCount), 0);
        for (int i = 0; i < s->textureCount; ++i) {
            if (!s->texPixels[i]) continue;
            RefTexture t; t.rgba8 = s->texPixels[i]; t.w = s->texW[i]; t.h = s->texH[i]; t.wrapV = 1;
            r.tex[static_cast<size_t>(i)] = registerTexture(t);
        }
        sv.texObjects = r.tex.data();
        sv.textureCount = s->textureCount;
        if (s->mrPixels) {
            r.texMr.assign(static_cast<size_t>(s->textureCount), 0);
            for (int i = 0; i < s->textureCount; ++i) {
                if (!s->mrPixels[i]) continue;
                RefTexture t; t.rgba8 = s->mrPixels[i]; t.w = s->mrW[i]; t.h = s->mrH[i]; t.wrapV = 1;
                r.texMr[static_cast<size_t>(i)] = registerTexture(t);
            }
            sv.texObjectsMr = r.texMr.data();
        }
    }
    sv.hasEnvMap = s->hasEnv != 0;
    if (s->hasEnv) {
        RefTexture t; t.f4 = s->envTexels; t.w = s->envW; t.h = s->envH; t.wrapV = 0;
        sv.envMap.texObj = registerTexture(t);
        sv.envMap.width = s->envW;
        sv.envMap.height = s->envH;
        sv.envMap.intensity = s->envIntensity;
        sv.envMap.rotationRadians = s->envRotation;
        sv.envMap.marginalCdf = const_cast<float*>(s->envMarginal);
        sv.envMap.conditionalCdf = const_cast<float*>(s->envConditional);
        sv.envMap.totalPower = s->envTotalPower;
    }
}

// closest hit through the oracle traversal, attributes as __closesthit__radiance
bool traceClosestRef(const OScene* s, const WfSceneView& sv, const Ray& ray, Intersection& its)
{
    const float r6[6] = {ray.origin.x, ray.origin.y, ray.origin.z, ray.direction.x, ray.direction.y, ray.direction.z};
    int tri = -1;
    float tuv[3] = {0, 0, 0};
    or_trace_closest(s, r6, 1, &tri, tuv);
    its.triangleIndex = -1;
    if (tri < 0) return false;
    const float u = tuv[1], v = tuv[2], w0 = 1.0f - u - v;
    const TriangleData T = sv.triangles[tri];
    const float t = tuv[0];
    const Float3 O = ray.origin, D = ray.direction;
    its.t = t;
    its.triangleIndex = tri;
    its.hitPoint = {O.x + t * D.x, O.y + t * D.y, O.z + t * D.z};
    its.hitNormal = normalize3({w0 * T.n0.x + u * T.n1.x + v * T.n2.x, w0 * T.n0.y + u * T.n1.y + v * T.n2.y,
                                w0 * T.n0.z + u * T.n1.z + v * T.n2.z});
    its.uv = {w0 * T.uv0.x + u * T.uv1.x + v * T.uv2.x, w0 * T.uv0.y + u * T.uv1.y + v * T.uv2.y};
    return true;
}

bool occludedRef(const OScene* s, const ShadowRayRecord& sr)
{
    const float r6[6] = {sr.origin.x, sr.origin.y, sr.origin.z, sr.direction.x, sr.direction.y, sr.direction.z};
    uint8_t occ = 0;
    or_trace_occluded(s, r6, &sr.tMax, 1, &occ);
    return occ != 0;
}

Float3 renderOne(const OScene* s, const WfSceneView& sv, const CameraData& cam, int W, int H, int maxDepth,
                 uint32_t pixel, uint32_t sampleIndex, int* hitLog, OStats* st, RngState* rngIO = nullptr)
{
    // ray_generate.cu:49-73 (pixel index == path slot; frameIndex == sample index)
    const int px = static_cast<int>(pixel % static_cast<uint32_t>(W));
    const int py = static_cast<int>(pixel / static_cast<uint32_t>(W));
    // rngIO: the megakernel's per-pixel stream carried from the previous path (optix_programs.cu:64-72)
    RngState rng = rngIO ? *rngIO : makeRng(hashUint(pixel ^ (sampleIndex * 0x9e3779b9u)));
    const float jx = rngNextFloat01(rng) - 0.5f;
    const float jy = rngNextFloat01(rng) - 0.5f;
    PathState ps;
    ps.ray = generatePrimaryRay(px, py, W, H, cam, jx, jy);
    ps.throughput = {1.f, 1.f, 1.f};
    ps.accumulatedColor = {0.f, 0.f, 0.f};
    ps.eta = 1.f;
    ps.brdfPDF = 0.f;
    ps.specularBounce = true;
    ps.bounceCount = 0;
    ps.pixelIndex = pixel;
    if (hitLog) for (int i = 0; i < maxDepth; ++i) hitLog[i] = -2;
    const DirectLightingContext ctx = makeDirectLightingContext(sv);

    while (ps.bounceCount < maxDepth) {
        // traceRay, rt_optix_shading.cuh:412-447
        Intersection its{};
        const bool hit = traceClosestRef(s, sv, ps.ray, its);
        if (st) st->extends++;
        if (hitLog) hitLog[ps.bounceCount] = its.triangleIndex;
        if (!hit) {
            accumulateEnvMapHit(ps, ctx);
            break;
        }
        BsdfData bsdf = loadBsdfForTriangle(ctx, sv.bsdfs, sv.triangleBsdfIds, its.triangleIndex, its.uv);
        if (ctx.triangleEmitterFlags[its.triangleIndex] != 0) accumulateEmitterHit(ps, its, ctx);
        if (bsdfIsDiffuse(bsdf)) {
            ps.specularBounce = false;
            {
                ShadowRayRecord sr{};
                if (prepareAreaEmitterNEE(ps, rng, its, bsdf, ctx, sr)) {
                    if (st) st->shadowRays++;
                    if (!occludedRef(s, sr)) ps.accumulatedColor = add3(ps.accumulatedColor, sr.contribution);
                }
            }
            for (int si = 0; si < ctx.spotlightCount; ++si) {
                ShadowRayRecord sr{};
                if (!prepareSpotlightNEE(ps, its, bsdf, ctx, si, sr)) continue;
                if (st) st->shadowRays++;
                if (!occludedRef(s, sr)) ps.accumulatedColor = add3(ps.accumulatedColor, sr.contribution);
            }
            {
                ShadowRayRecord sr{};
                if (prepareEnvMapNEE(ps, rng, its, bsdf, ctx, sr)) {
                    if (st) st->shadowRays++;
                    if (!occludedRef(s, sr)) ps.accumulatedColor = add3(ps.accumulatedColor, sr.contribution);
                }
            }
        } else {
            ps.specularBounce = true;
        }
        scatterPath(ps, rng, its, bsdf);
        if (!russianRoulette(ps, rng)) break;
        ps.bounceCount++;
    }
    if (rngIO) *rngIO = rng;
    return ps.accumulatedColor;
}
}  // namespace

// ---------------------------------------------------------------------------
// exported entry points
// ---------------------------------------------------------------------------
REF_API uint32_t ref_hash_uint(uint32_t x) { return hashUint(x); }

REF_API void ref_rng_stream(uint32_t seed, int n, uint32_t* outU32, float* outF)
{
    RngState a = makeRng(seed), b = makeRng(seed);
    for (int i = 0; i < n; ++i) {
        if (outU32) outU32[i] = rngNextU32(a);
        if (outF) outF[i] = rngNextFloat01(b);
    }
}

REF_API void ref_bsdf_eval(const OBsdf* b, const float* wi, const float* wo, float* out, int n)
{
    const BsdfData& bd = *reinterpret_cast<const BsdfData*>(b);
    for (int i = 0; i < n; ++i) {
        BsdfQueryRecord r{};
        r.wi = {wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        r.wo = {wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]};
        r.measure = BSDF_ESolidAngle;
        const Float3 v = bsdfEval(bd, r);
        out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
    }
}

REF_API void ref_bsdf_pdf(const OBsdf* b, const float* wi, const float* wo, float* out, int n)
{
    const BsdfData& bd = *reinterpret_cast<const BsdfData*>(b);
    for (int i = 0; i < n; ++i) {
        BsdfQueryRecord r{};
        r.wi = {wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        r.wo = {wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]};
        r.measure = BSDF_ESolidAngle;
        out[i] = bsdfPdf(bd, r);
    }
}

REF_API void ref_bsdf_sample(const OBsdf* b, const float* wi, const float* u, float* outWo, float* outWeight,
                             float* outPdf, float* outEta, int n)
{
    const BsdfData& bd = *reinterpret_cast<const BsdfData*>(b);
    for (int i = 0; i < n; ++i) {
        BsdfQueryRecord r{};
        r.wi = {wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        r.rndExtra = u[3 * i];
        const Float3 w = bsdfSample(bd, r, u[3 * i + 1], u[3 * i + 2]);
        outWo[3 * i] = r.wo.x; outWo[3 * i + 1] = r.wo.y; outWo[3 * i + 2] = r.wo.z;
        outWeight[3 * i] = w.x; outWeight[3 * i + 1] = w.y; outWeight[3 * i + 2] = w.z;
        outPdf[i] = bsdfPdf(bd, r);
        outEta[i] = r.eta;
    }
}

REF_API void ref_env_eval(const OScene* s, const float* dirs, float* out, int n)
{
    RefScene rs; buildRefScene(s, rs);
    for (int i = 0; i < n; ++i) {
        const Float3 r = envMapEval(rs.sv.envMap, {dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]});
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
}

REF_API void ref_env_pdf(const OScene* s, const float* dirs, float* out, int n)
{
    RefScene rs; buildRefScene(s, rs);
    for (int i = 0; i < n; ++i) out[i] = envMapPdf(rs.sv.envMap, {dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]});
}

REF_API void ref_env_sample(const OScene* s, const float* u, float* outDir, float* outPdf, float* outRad, int n)
{
    RefScene rs; buildRefScene(s, rs);
    for (int i = 0; i < n; ++i) {
        const EnvMapSampleResult r = envMapSample(rs.sv.envMap, u[2 * i], u[2 * i + 1]);
        outDir[3 * i] = r.direction.x; outDir[3 * i + 1] = r.direction.y; outDir[3 * i + 2] = r.direction.z;
        outPdf[i] = r.pdf;
        outRad[3 * i] = r.radiance.x; outRad[3 * i + 1] = r.radiance.y; outRad[3 * i + 2] = r.radiance.z;
    }
}

REF_API void ref_render_samples(const OScene* s, const OCamera* cam, const OConfig* cfg, const uint32_t* pixels,
                                const uint32_t* sampleIndices, int n, float* outRadiance, int* hitLog, OStats* stats,
                                int threads)
{
    RefScene rs; buildRefScene(s, rs);
    const CameraData& c = *reinterpret_cast<const CameraData*>(cam);
    int64_t ext = 0, sh = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) reduction(+ : ext, sh)
#endif
    for (int i = 0; i < n; ++i) {
        OStats local{0, 0};
        const Float3 L = renderOne(s, rs.sv, c, cfg->width, cfg->height, cfg->maxDepth, pixels[i], sampleIndices[i],
                                   hitLog ? hitLog + static_cast<size_t>(i) * cfg->maxDepth : nullptr, &local);
        outRadiance[3 * i] = L.x; outRadiance[3 * i + 1] = L.y; outRadiance[3 * i + 2] = L.z;
        ext += local.extends; sh += local.shadowRays;
    }
    (void)threads;
    if (stats) { stats->extends += ext; stats->shadowRays += sh; }
}

// one megakernel frame, optix_programs.cu:54-99: per pixel one stream through spp paths, summed with add3 and
// scaled with div3 (the reference's own helpers)
REF_API void ref_render_megakernel(const OScene* s, const OCamera* cam, const OConfig* cfg, const uint32_t* pixels,
                                   int n, uint32_t frameIndex, int spp, float* outMean, OStats* stats, int threads)
{
    RefScene rs; buildRefScene(s, rs);
    const CameraData& c = *reinterpret_cast<const CameraData*>(cam);
    int64_t ext = 0, sh = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) reduction(+ : ext, sh)
#endif
    for (int i = 0; i < n; ++i) {
        OStats local{0, 0};
        RngState rng = makeRng(hashUint(pixels[i] ^ (frameIndex * 0x9e3779b9u)));
        Float3 sum = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < spp; ++k)
            sum = add3(sum, renderOne(s, rs.sv, c, cfg->width, cfg->height, cfg->maxDepth, pixels[i], 0u, nullptr,
                                      &local, &rng));
        const Float3 m = div3(sum, static_cast<float>(spp));
        outMean[3 * i] = m.x; outMean[3 * i + 1] = m.y; outMean[3 * i + 2] = m.z;
        ext += local.extends; sh += local.shadowRays;
    }
    (void)threads;
    if (stats) { stats->extends += ext; stats->shadowRays += sh; }
}

// present: ray_present.cu:43-62 over a [count] radiance buffer (frameIndex = samples so far)
REF_API void ref_present(float* accum, const float* radiance, int count, uint32_t frameIndex, uint32_t* outRGBA8)
{
    Float3* a = reinterpret_cast<Float3*>(accum);
    const Float3* x = reinterpret_cast<const Float3*>(radiance);
    for (int i = 0; i < count; ++i) {
        const Float3 blended = accumulateWelford(a, static_cast<uint32_t>(i), x[i], frameIndex);
        if (outRGBA8) outRGBA8[i] = packPixelGamma(blended);
    }
}

REF_API int ref_rr_start(void) { return 3; }   // rt_path_integrator.cuh:56 (compile-time in the reference)
