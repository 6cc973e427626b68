/*
 * oracle/ref_layout_fields.h -- ORACLE (test infrastructure only).
 *
 * Field lists of the reference's LaunchParams (include/optix_launch_params.h:34-86),
 * WavefrontSoA and WfSceneView (include/wavefront/wavefront_buffers.h:40-121) and
 * EnvMapData (include/render_kernel.h:68-77).  ref_layout.cpp expands them twice,
 * once over the reference's headers and once over include/bte/launch_params.h, and
 * the test compares every offset and size.
 */
#define BTE_ENVMAP_FIELDS(X) X(EnvMapData, texObj) X(EnvMapData, width) X(EnvMapData, height) \
    X(EnvMapData, intensity) X(EnvMapData, rotationRadians) X(EnvMapData, marginalCdf) \
    X(EnvMapData, conditionalCdf) X(EnvMapData, totalPower)
#define BTE_SOA_FIELDS(X) X(WavefrontSoA, rayOrigin) X(WavefrontSoA, rayDir) X(WavefrontSoA, throughput) \
    X(WavefrontSoA, radiance) X(WavefrontSoA, eta) X(WavefrontSoA, brdfPDF) X(WavefrontSoA, specularBounce) \
    X(WavefrontSoA, bounceCount) X(WavefrontSoA, pixelIndex) X(WavefrontSoA, rngState) X(WavefrontSoA, hitTriIndex) \
    X(WavefrontSoA, hitPoint) X(WavefrontSoA, hitNormal) X(WavefrontSoA, hitUV) X(WavefrontSoA, rayQueue) \
    X(WavefrontSoA, rayQueueNext) X(WavefrontSoA, rayCount) X(WavefrontSoA, rayCountNext) X(WavefrontSoA, shadowCount) \
    X(WavefrontSoA, shadowOrigin) X(WavefrontSoA, shadowDir) X(WavefrontSoA, shadowTMax) X(WavefrontSoA, shadowContrib) \
    X(WavefrontSoA, shadowPathIdx) X(WavefrontSoA, maxPaths) X(WavefrontSoA, maxShadows)
#define BTE_VIEW_FIELDS(X) X(WfSceneView, triangles) X(WfSceneView, triangleCount) \
    X(WfSceneView, triangleEmitterFlags) X(WfSceneView, triangleEmission) X(WfSceneView, bsdfs) \
    X(WfSceneView, bsdfCount) X(WfSceneView, triangleBsdfIds) X(WfSceneView, triangleMaterialIds) \
    X(WfSceneView, emitters) X(WfSceneView, emitterCount) X(WfSceneView, emitterTriIndices) \
    X(WfSceneView, emitterTriCdf) X(WfSceneView, sceneEmitterCdf) X(WfSceneView, spotlights) \
    X(WfSceneView, spotlightCount) X(WfSceneView, texObjects) X(WfSceneView, texObjectsMr) \
    X(WfSceneView, textureCount) X(WfSceneView, envMap) X(WfSceneView, hasEnvMap) X(WfSceneView, accumBuffer) \
    X(WfSceneView, frameIndex)
#define BTE_LP_FIELDS(X) X(LaunchParams, framebuffer) X(LaunchParams, accumBuffer) X(LaunchParams, width) \
    X(LaunchParams, height) X(LaunchParams, launchOffsetY) X(LaunchParams, frameIndex) X(LaunchParams, camera) \
    X(LaunchParams, handle) X(LaunchParams, triangles) X(LaunchParams, triangleCount) X(LaunchParams, bsdfs) \
    X(LaunchParams, bsdfCount) X(LaunchParams, triangleBsdfIds) X(LaunchParams, triangleMaterialIds) \
    X(LaunchParams, triangleEmitterFlags) X(LaunchParams, triangleEmission) X(LaunchParams, emitters) \
    X(LaunchParams, emitterCount) X(LaunchParams, emitterTriIndices) X(LaunchParams, emitterTriCdf) \
    X(LaunchParams, sceneEmitterCdf) X(LaunchParams, spotlights) X(LaunchParams, spotlightCount) \
    X(LaunchParams, texObjects) X(LaunchParams, texObjectsMr) X(LaunchParams, textureCount) X(LaunchParams, envMap) \
    X(LaunchParams, hasEnvMap) X(LaunchParams, wf)
#define BTE_LAYOUT_ALL(X) BTE_ENVMAP_FIELDS(X) BTE_SOA_FIELDS(X) BTE_VIEW_FIELDS(X) BTE_LP_FIELDS(X)

#define BTE_LAYOUT_OFFSET(T, f) (long long)offsetof(T, f), (long long)sizeof(((T*)0)->f),
#define BTE_LAYOUT_TABLE { BTE_LAYOUT_ALL(BTE_LAYOUT_OFFSET) (long long)sizeof(EnvMapData), \
    (long long)sizeof(WavefrontSoA), (long long)sizeof(WfSceneView), (long long)sizeof(LaunchParams) }
