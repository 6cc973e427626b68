// bte_internal.h -- host-side shared declarations of libbte_b200.
#pragma once

#include "../../include/bte/render_api.h"

#include <string>
#include <vector>

namespace bte {

// Flattened scene as produced by the scene.xml/OBJ loader (bte_scene.cpp).
struct SceneData {
    std::vector<TriangleData> triangles;
    std::vector<Float3> materials;
    std::vector<int> triangleMaterialIds, triangleBsdfIds;
    std::vector<BsdfData> bsdfs;
    std::vector<Float3> triangleEmission;
    std::vector<uint8_t> triangleEmitterFlags;
    std::vector<EmitterData> emitters;
    std::vector<int> emitterTriIndices;
    std::vector<float> emitterTriCdf, sceneEmitterCdf;
    std::vector<SpotlightData> spotlights;
    std::vector<float> envRGBA;
    int envWidth = 0, envHeight = 0;
    float envIntensity = 1.0f, envRotationDeg = 0.0f;
    CameraData camera{};
    int width = 0, height = 0;
    // per material: RGBA8 albedo and metallic-roughness images (empty: none), as
    // src/main.cpp:603-612 builds them for cudaInitTextures / cudaInitMrTextures
    std::vector<std::vector<uint8_t>> albedoImages, mrImages;
    std::vector<int> albedoWidths, albedoHeights, mrWidths, mrHeights;
};

int sceneLoad(const char* path, SceneData& out, std::string& err);

// PNG / JPEG file or bytes -> RGBA8 rows top to bottom (bte_image.cpp); false with `err` on failure.
bool decodeImageRGBA8(const uint8_t* data, size_t size, std::vector<uint8_t>& rgba, int& width, int& height,
                      int& channelsInFile, std::string& err);
bool loadImageRGBA8(const std::string& path, std::vector<uint8_t>& rgba, int& width, int& height, int& channelsInFile,
                    std::string& err);
// A 16-bit PNG as 4 channels of 16-bit samples, little-endian bytes (false for any other image).
bool decodeImageRGBA16(const uint8_t* data, size_t size, std::vector<uint8_t>& rgba16le);

// glTF / GLB model flattened as the reference's loadGltfModel does (bte_gltf.cpp).
struct GltfSlot {
    BsdfData bsdf{};
    std::vector<uint8_t> albedo, mr;   // RGBA8, empty when none
    int albedoWidth = 0, albedoHeight = 0, mrWidth = 0, mrHeight = 0;
    Float3 emission{0.0f, 0.0f, 0.0f};
    bool isEmitter = false;
};
struct GltfResult {
    std::vector<TriangleData> triangles;
    std::vector<int> materialIds;   // per triangle, into materials
    std::vector<GltfSlot> materials;
    int skippedOutliers = 0;
};
// xf: posX/Y/Z, rotX/Y/Z (degrees), scaleX/Y/Z of the <model> element
bool loadGltf(const std::string& path, const float xf[9], GltfResult& out, std::string& err);

void setError(const std::string& msg);

}  // namespace bte
