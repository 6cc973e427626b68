// bte/render_kernel.h -- the reference's renderer API (include/render_kernel.h:96-211 of
// the reference) with C++ linkage, implemented over the C-ABI of bte/render_api.h.
//
// Drop-in for callers of the reference: same names, argument types and meaning.
// Like the reference (src/host/cuda_check.h:14-32) an error prints the library's
// message with the function name and terminates the process with EXIT_FAILURE.
// The OpenGL pixel buffer of cudaRegisterPBO does not exist on a headless B200;
// render into a device buffer registered with cudaSetOutputBuffer instead (or
// read the frame back with bte_read_framebuffer).
#pragma once

#include "render_api.h"

#include <cstdint>

void cudaInitOptix();   // builds the LBVH (no OptiX)
void cudaInitScene(const TriangleData* triangles, int triangleCount, const Float3* materials, int materialCount,
                   const int* triangleMaterialIds, int imageWidth, int imageHeight);
void cudaInit(const TriangleData& tri, const Float3& color, int imageWidth, int imageHeight);
void cudaInitCamera(const CameraData& camera);
void cudaInitTriangleEmission(const Float3* triangleEmission, int triangleCount);
void cudaInitTriangleEmitterFlags(const uint8_t* flags, int triangleCount);
void cudaInitEmitterTable(const EmitterData* emitters, int emitterCount, const int* emitterTriIndices,
                          int emitterTriIndexCount, const float* emitterTriCdf, int emitterTriCdfCount,
                          const float* sceneEmitterCdf);
void cudaInitBsdfs(const BsdfData* bsdfs, int bsdfCount, const int* triangleBsdfIds, int triangleCount);
void cudaInitSpotlights(const SpotlightData* spotlights, int spotlightCount);
void cudaInitTextures(const uint8_t* const* pixels, const int* widths, const int* heights, int textureCount);
void cudaInitMrTextures(const uint8_t* const* pixels, const int* widths, const int* heights, int textureCount);
void cudaInitEnvMap(const float* hdriPixelsRGBA, int width, int height, float intensity, float rotationDeg);
void cudaRegisterPBO(uint32_t pbo);
void cudaSetOutputBuffer(uint32_t* deviceRGBA8);
void cudaResetAccumulation(int imageWidth, int imageHeight);
void cudaRender(int imageWidth, int imageHeight);
bool cudaToggleDenoiser();

enum class RenderMode {
    Megakernel,
    Wavefront,
};
void cudaSetRenderMode(RenderMode mode);
RenderMode cudaGetRenderMode();
void cudaCleanup();
