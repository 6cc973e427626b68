/*
 * bte_oracle.h -- ORACLE (test infrastructure only; never linked into the
 * product).  CPU restatement of Blue Truth Engine's wavefront path-tracing
 * hot path, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker.
 *
 * Parity pin: compiled with -DBTE_ORACLE_LIBM the oracle calls glibc's
 * sinf/cosf/... exactly where the reference calls them, and is compared
 * bit-for-bit with the reference's own shading headers compiled on the host
 * (oracle/ref_harness.cpp -> oracle/_ref/libbteref.so).  Compiled without it,
 * the oracle uses bte_oracle_math.h, the same double-evaluated elementary
 * functions the CUDA kernels use, and is compared bit-for-bit with the GPU.
 *
 * All struct layouts are byte-identical to the reference's POD types
 * (include/render_kernel.h:9-94 in the reference).
 */
#ifndef BTE_ORACLE_H
#define BTE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y; } OF2;
typedef struct { float x, y, z; } OF3;
typedef struct { float x, y, z, w; } OF4;

/* render_kernel.h:22-26 */
typedef struct { OF3 v0, v1, v2; OF3 n0, n1, n2; OF2 uv0, uv1, uv2; } OTri;
/* render_kernel.h:33-40 */
typedef struct { OF3 origin, forward, right, up; float fovYRadians, aspect; } OCamera;
/* render_kernel.h:44-51 */
typedef struct { int triIndexOffset, triCount, cdfOffset; OF3 radiance; float areaSum, powerWeight; } OEmitter;
/* render_kernel.h:56-63 */
typedef struct { OF3 position, direction, radiance; float intensity, innerConeCosine, outerConeCosine; } OSpot;
/* render_kernel.h:88-94 */
typedef struct { int type; OF4 p0, p1, p2, p3; } OBsdf;

enum { O_BSDF_DIFFUSE = 1, O_BSDF_DIELECTRIC = 2, O_BSDF_MIRROR = 3, O_BSDF_MICROFACET = 4, O_BSDF_DISNEY = 5 };

/* env-map sampling modes */
enum { O_ENV_CDF = 0, O_ENV_ALIAS = 1 };

/* Flattened scene, all arrays caller-owned (the same arrays the renderer's
 * bte_init_* calls receive). */
typedef struct {
    const OTri* triangles; int triangleCount;
    const uint8_t* emitterFlags;          /* [T] */
    const OF3* emission;                  /* [T] */
    const OBsdf* bsdfs; int bsdfCount;
    const int* triBsdfIds;                /* [T] */
    const int* triMaterialIds;            /* [T] or NULL */
    const OEmitter* emitters; int emitterCount;
    const int* emitterTriIndices;
    const float* emitterTriCdf;
    const float* sceneEmitterCdf;         /* [E+1] */
    const OSpot* spots; int spotCount;
    /* material textures (RGBA8, wrap/wrap, bilinear, normalized float) */
    const uint8_t* const* texPixels; const int* texW; const int* texH; int textureCount;
    const uint8_t* const* mrPixels; const int* mrW; const int* mrH;
    /* environment map (float4 texels, wrap u / clamp v, bilinear) */
    int hasEnv;
    const float* envTexels; int envW, envH;
    float envIntensity, envRotation;      /* rotation in radians */
    const float* envMarginal;             /* [H+1]      (CDF mode) */
    const float* envConditional;          /* [H*(W+1)]  (CDF mode) */
    float envTotalPower;
    int envSampling;                      /* O_ENV_CDF | O_ENV_ALIAS */
    const float* aliasRowProb; const int* aliasRowIdx;   /* [H] */
    const float* aliasColProb; const int* aliasColIdx;   /* [H*W] */
    const float* envPixelPdf;                            /* [H*W] discrete pdf */
    /* CPU acceleration structure built by or_build_accel (NULL: brute force) */
    void* accel;
} OScene;

typedef struct {
    int width, height;
    int maxDepth;          /* extend+shade steps per path (reference: MAX_BOUNCES) */
    int rrStart;           /* roulette applies when bounceCount > rrStart (reference: 3) */
} OConfig;

typedef struct {
    int64_t extends;       /* closest-hit rays traced */
    int64_t shadowRays;    /* shadow rays generated (prepare*NEE returned true) */
} OStats;

/* ---- unit-level restatements (known-answer tests) ---- */
uint32_t or_hash_uint(uint32_t x);
void or_rng_stream(uint32_t seed, int n, uint32_t* outU32, float* outF);
void or_math_eval(int fn, const float* a, const float* b, float* out, int n);

/* mode: 0 eval (out3), 1 pdf (out1), 2 sample (wo3 + weight3 + pdf1 + eta1) */
void or_bsdf_eval(const OBsdf* b, const float* wi, const float* wo, float* out, int n);
void or_bsdf_pdf(const OBsdf* b, const float* wi, const float* wo, float* out, int n);
void or_bsdf_sample(const OBsdf* b, const float* wi, const float* u /*[n*3]: rndExtra,u1,u2*/,
                    float* outWo, float* outWeight, float* outPdf, float* outEta, int n);

void or_env_build_cdf(const float* rgba, int w, int h, float* marginal, float* conditional, float* totalPower);
void or_env_build_alias(const float* rgba, int w, int h,
                        float* rowProb, int* rowIdx, float* colProb, int* colIdx, float* pixelPdf,
                        double* totalPowerD);
void or_env_eval(const OScene* s, const float* dirs, float* out, int n);
void or_env_pdf(const OScene* s, const float* dirs, float* out, int n);
void or_env_sample(const OScene* s, const float* u, float* outDir, float* outPdf, float* outRad, int n);
void or_tex_float4(const float* texels, int w, int h, int wrapV, const float* uv, float* out, int n);
void or_tex_sample_f4(const float* texels, int w, int h, int wrapV, float u, float v, float out[4]);
void or_tex_sample_rgba8(const uint8_t* px, int w, int h, float u, float v, float out[4]);

/* ---- traversal ---- */
int  or_build_accel(OScene* s);          /* CPU BVH for large scenes */
void or_free_accel(OScene* s);
/* rays: [n*6] origin, dir.  out: triIdx[n], t/u/v [n*3].  tmin = 1e-4, tmax = 1e30 */
void or_trace_closest(const OScene* s, const float* rays, int n, int* outTri, float* outTuv);
void or_trace_occluded(const OScene* s, const float* rays, const float* tmax, int n, uint8_t* outOcc);

/* ---- full paths ----
 * Traces the paths of `n` (pixel, sampleIndex) pairs in the reference's
 * canonical (megakernel) order and writes each sample's radiance [n*3].
 * hitLog (optional, [n*maxDepth]) receives the closest-hit triangle index of
 * every extend (-1 miss, -2 not traced).  stats (optional) accumulates counts. */
void or_render_samples(const OScene* s, const OCamera* cam, const OConfig* cfg,
                       const uint32_t* pixels, const uint32_t* sampleIndices, int n,
                       float* outRadiance, int* hitLog, OStats* stats, int threads);
/* one megakernel frame (src/optix_programs.cu:54-108): per pixel one RNG stream through spp paths; the frame's
 * mean radiance per pixel [n*3] */
void or_render_megakernel(const OScene* s, const OCamera* cam, const OConfig* cfg, const uint32_t* pixels, int n,
                          uint32_t frameIndex, int spp, float* outMean, OStats* stats, int threads);

void or_path_rays(const OScene* s, const OCamera* cam, const OConfig* cfg, uint32_t pixel, uint32_t sampleIndex,
                  float* rays, int* hits);

/* Welford running mean (FP32, rt_path_integrator.cuh:72-87) and gamma pack (:93-105). */
void or_present(float* accum, const float* radiance, int count, uint32_t frameIndex, uint32_t* outRGBA8);
uint32_t or_pack_gamma(float r, float g, float b);

int or_math_mode(void);                  /* 1 = glibc (pin build), 0 = portable */

#ifdef __cplusplus
}
#endif
#endif
