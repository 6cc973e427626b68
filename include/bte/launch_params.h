/*
 * bte/launch_params.h -- the reference's per-frame launch-parameter block and wavefront
 * state layout, byte for byte (include/optix_launch_params.h:34-86 and
 * include/wavefront/wavefront_buffers.h:40-121 of the reference), for code written
 * against those structs.
 *
 * The only change of type is LaunchParams.handle: the reference's
 * OptixTraversableHandle (an unsigned 64-bit integer) is a uint64_t here and holds the
 * device address of this library's BVH (8-wide nodes, or binary nodes when the
 * 8-wide tree is off).  Texture handles (cudaTextureObject_t, an unsigned 64-bit
 * integer) stay 64-bit integers.  Offsets assume the LP64 ABI the reference is built
 * for; the static assertions below pin every offset, and a host program compiled
 * from the reference's own headers checks them field by field (oracle/).
 *
 * bte_get_launch_params fills one LaunchParams with the current frame's device
 * pointers and sizes.  Fields whose data this library keeps in another form are
 * documented there (textures are filtered in software, so there are no texture
 * objects; the wavefront state is packed float4 records, so only the queue and
 * counter pointers of WavefrontSoA point at live data).
 */
#ifndef BTE_LAUNCH_PARAMS_H
#define BTE_LAUNCH_PARAMS_H

#include "render_api.h"

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* render_kernel.h:68-77 */
typedef struct {
    unsigned long long texObj;   /* cudaTextureObject_t; 0 here (texels are read by software filtering) */
    int width, height;
    float intensity;
    float rotationRadians;
    float* marginalCdf;          /* [height+1] */
    float* conditionalCdf;       /* [height*(width+1)] */
    float totalPower;
} EnvMapData;

/* include/wavefront/wavefront_buffers.h:40-90 */
typedef struct {
    Float3* rayOrigin;
    Float3* rayDir;
    Float3* throughput;
    Float3* radiance;
    float* eta;
    float* brdfPDF;
    unsigned char* specularBounce;
    int* bounceCount;
    uint32_t* pixelIndex;
    uint32_t* rngState;
    int* hitTriIndex;
    Float3* hitPoint;
    Float3* hitNormal;
    Float2* hitUV;
    int* rayQueue;
    int* rayQueueNext;
    int* rayCount;
    int* rayCountNext;
    int* shadowCount;
    Float3* shadowOrigin;
    Float3* shadowDir;
    float* shadowTMax;
    Float3* shadowContrib;
    uint32_t* shadowPathIdx;
    int maxPaths;
    int maxShadows;
} WavefrontSoA;

/* include/wavefront/wavefront_buffers.h:98-121 */
typedef struct {
    const TriangleData* triangles;
    int triangleCount;
    const uint8_t* triangleEmitterFlags;
    const Float3* triangleEmission;
    const BsdfData* bsdfs;
    int bsdfCount;
    const int* triangleBsdfIds;
    const int* triangleMaterialIds;
    const EmitterData* emitters;
    int emitterCount;
    const int* emitterTriIndices;
    const float* emitterTriCdf;
    const float* sceneEmitterCdf;
    const SpotlightData* spotlights;
    int spotlightCount;
    const unsigned long long* texObjects;     /* const cudaTextureObject_t* */
    const unsigned long long* texObjectsMr;
    int textureCount;
    EnvMapData envMap;
    bool hasEnvMap;
    Float3* accumBuffer;
    int frameIndex;
} WfSceneView;

/* include/optix_launch_params.h:34-86 */
typedef struct {
    uint32_t* framebuffer;
    Float3* accumBuffer;
    int width;
    int height;
    int launchOffsetY;
    uint32_t frameIndex;
    CameraData camera;
    uint64_t handle;                          /* OptixTraversableHandle -> BVH device address */
    const TriangleData* triangles;
    int triangleCount;
    const BsdfData* bsdfs;
    int bsdfCount;
    const int* triangleBsdfIds;
    const int* triangleMaterialIds;
    const uint8_t* triangleEmitterFlags;
    const Float3* triangleEmission;
    const EmitterData* emitters;
    int emitterCount;
    const int* emitterTriIndices;
    const float* emitterTriCdf;
    const float* sceneEmitterCdf;
    const SpotlightData* spotlights;
    int spotlightCount;
    const unsigned long long* texObjects;     /* const cudaTextureObject_t* */
    const unsigned long long* texObjectsMr;
    int textureCount;
    EnvMapData envMap;
    bool hasEnvMap;
    WavefrontSoA wf;
} LaunchParams;

/*
 * Fills *out with the current scene's and frame's device pointers and sizes
 * (the block the reference's render_kernel.cu:58-143 and wavefront_host.cu:122-148
 * build before each launch).  Valid until the next upload, resize or cleanup.
 *   framebuffer / accumBuffer: the packed RGBA8 frame and the FP32 running mean
 *     (W*H*3 floats); width/height/frameIndex as accumulated so far;
 *     launchOffsetY is 0 (frames are never split into row bands).
 *   handle: device address of the BVH nodes; triangles .. spotlights: the uploaded
 *     arrays (device copies).
 *   texObjects / texObjectsMr: NULL (textures are RGBA8 images filtered in
 *     software); textureCount: the number of albedo textures uploaded.
 *   envMap: texObj 0, sizes, intensity, rotation in radians, the CDF tables and
 *     their total; hasEnvMap.
 *   wf: rayQueue / rayQueueNext: the two path-index queues; rayCount: the
 *     per-bounce ray counters (maxDepth+1 ints, bounce b at rayCount[b]);
 *     rayCountNext = rayCount + 1; shadowCount: the per-bounce shadow-ray
 *     counters; maxPaths: paths of the last frame; maxShadows: maxPaths times the
 *     shadow slots per path.  The path state lives in packed float4 records, not
 *     in the reference's per-field arrays, so every other pointer is NULL.
 * No reference counterpart as a function (the reference fills the block internally).
 */
int bte_get_launch_params(LaunchParams* out);

#ifdef __cplusplus
}  /* extern "C" */
#define BTE_LP_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define BTE_LP_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

/* LP64 layout of the reference's structs (checked against the reference's headers by oracle/ref_layout_*). */
BTE_LP_STATIC_ASSERT(sizeof(EnvMapData) == 48, "EnvMapData size");
BTE_LP_STATIC_ASSERT(offsetof(EnvMapData, marginalCdf) == 24 && offsetof(EnvMapData, totalPower) == 40,
                     "EnvMapData offsets");
BTE_LP_STATIC_ASSERT(sizeof(WavefrontSoA) == 200, "WavefrontSoA size");
BTE_LP_STATIC_ASSERT(offsetof(WavefrontSoA, hitTriIndex) == 80 && offsetof(WavefrontSoA, rayQueue) == 112 &&
                     offsetof(WavefrontSoA, shadowOrigin) == 152 && offsetof(WavefrontSoA, maxPaths) == 192,
                     "WavefrontSoA offsets");
BTE_LP_STATIC_ASSERT(sizeof(WfSceneView) == 216, "WfSceneView size");
BTE_LP_STATIC_ASSERT(offsetof(WfSceneView, envMap) == 144 && offsetof(WfSceneView, hasEnvMap) == 192 &&
                     offsetof(WfSceneView, accumBuffer) == 200 && offsetof(WfSceneView, frameIndex) == 208,
                     "WfSceneView offsets");
BTE_LP_STATIC_ASSERT(sizeof(LaunchParams) == 496, "LaunchParams size");
BTE_LP_STATIC_ASSERT(offsetof(LaunchParams, camera) == 32 && offsetof(LaunchParams, handle) == 88 &&
                     offsetof(LaunchParams, triangles) == 96 && offsetof(LaunchParams, emitters) == 160 &&
                     offsetof(LaunchParams, texObjects) == 216 && offsetof(LaunchParams, envMap) == 240 &&
                     offsetof(LaunchParams, hasEnvMap) == 288 && offsetof(LaunchParams, wf) == 296,
                     "LaunchParams offsets");

#endif /* BTE_LAUNCH_PARAMS_H */
