/*
 * oracle/ref_gltf.cpp -- ORACLE (test infrastructure only).
 *
 * glTF pin: the reference's own src/gltf_loader.cpp, compiled where it lies with
 * its vendored tinygltf and stb_image, against the GLM shim in ref_shim/glm
 * (GLM is not in this tree).  refg_load runs loadGltfModel on a file and the
 * accessors copy its result out for comparison with the product's reader.
 * Built by oracle/Makefile into oracle/_ref/libbteref_gltf.so.
 */
#define STB_IMAGE_IMPLEMENTATION
#include "stb_image.h"

#include "gltf_loader.h"

#include <cstring>

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
GltfLoadResult g_res;
}

// xf: posX/Y/Z, rotX/Y/Z (degrees), scaleX/Y/Z; returns the triangle count
REF_API int refg_load(const char* path, const float* xf)
{
    TransformDesc t;
    t.posX = xf[0]; t.posY = xf[1]; t.posZ = xf[2];
    t.rotXDegrees = xf[3]; t.rotYDegrees = xf[4]; t.rotZDegrees = xf[5];
    t.scaleX = xf[6]; t.scaleY = xf[7]; t.scaleZ = xf[8];
    g_res = loadGltfModel(path, t);
    return (int)g_res.triangles.size();
}

REF_API int refg_material_count(void) { return (int)g_res.materials.size(); }

REF_API void refg_triangles(TriangleData* tris, int* matIds)
{
    std::memcpy(tris, g_res.triangles.data(), g_res.triangles.size() * sizeof(TriangleData));
    std::memcpy(matIds, g_res.materialIds.data(), g_res.materialIds.size() * sizeof(int));
}

// bsdf, emission[3], isEmitter; image sizes (0 when none); images copied when the pointers are non-null
REF_API void refg_material(int i, BsdfData* bsdf, float* emission, int* isEmitter, int* albedoWH, int* mrWH,
                           uint8_t* albedo, uint8_t* mr)
{
    const GltfMaterialSlot& s = g_res.materials[(size_t)i];
    *bsdf = s.bsdf;
    emission[0] = s.emission.x; emission[1] = s.emission.y; emission[2] = s.emission.z;
    *isEmitter = s.isEmitter ? 1 : 0;
    albedoWH[0] = s.albedo.pixels.empty() ? 0 : s.albedo.width;
    albedoWH[1] = s.albedo.pixels.empty() ? 0 : s.albedo.height;
    mrWH[0] = s.metallicRoughness.pixels.empty() ? 0 : s.metallicRoughness.width;
    mrWH[1] = s.metallicRoughness.pixels.empty() ? 0 : s.metallicRoughness.height;
    if (albedo && !s.albedo.pixels.empty()) std::memcpy(albedo, s.albedo.pixels.data(), s.albedo.pixels.size());
    if (mr && !s.metallicRoughness.pixels.empty())
        std::memcpy(mr, s.metallicRoughness.pixels.data(), s.metallicRoughness.pixels.size());
}
