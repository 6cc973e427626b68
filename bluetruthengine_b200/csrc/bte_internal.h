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
};

int sceneLoad(const char* path, SceneData& out, std::string& err);

void setError(const std::string& msg);

}  // namespace bte
