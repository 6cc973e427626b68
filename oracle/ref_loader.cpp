/*
 * oracle/ref_loader.cpp -- ORACLE (test infrastructure only).
 *
 * Loader pin: the reference's own scene.xml parser (src/scene.cpp, compiled
 * where it lies), its vendored OBJ parser (external/tinyobjloader) and its
 * transforms (include/mesh_transform.h), glued as src/main.cpp:267-401 and
 * :629-758 flatten a scene (that glue is restated here because main.cpp also
 * pulls in the window/GL stack).  Produces the flattened triangle, BSDF and
 * emitter arrays for comparison with the product's loader, and per material
 * the texture colour and RGBA8 image of loadTextureAverage / loadImageRGBA
 * (src/main.cpp:407-470) through the reference's vendored stb_image.  <model>
 * entries go through the reference's own loadGltfModel (src/gltf_loader.cpp,
 * linked in with the GLM shim) and the merge of src/main.cpp:760-817.
 * Built by oracle/Makefile into oracle/_ref/libbteref_loader.so.
 */
#include "scene.h"
#include "mesh_transform.h"
#include "gltf_loader.h"
#define TINYOBJLOADER_IMPLEMENTATION
#include "tiny_obj_loader.h"
#define STB_IMAGE_IMPLEMENTATION
#include "stb_image.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
std::vector<TriangleData> g_tris;
std::vector<BsdfData> g_bsdfs;
std::vector<int> g_triBsdf, g_triMat, g_emTri;
std::vector<float> g_emCdf, g_sceneCdf, g_cam;
std::vector<uint8_t> g_flags;
std::vector<float> g_matColour;                 // 3 per material
std::vector<std::vector<uint8_t>> g_matImage;   // RGBA8 per material (empty: none)
std::vector<int> g_matW, g_matH;
std::vector<std::vector<uint8_t>> g_matMr;      // metallic-roughness RGBA8 per material (empty: none)
std::vector<int> g_mrW, g_mrH;
int g_emitterCount = 0;
std::vector<EmitterData> g_emitters;            // src/main.cpp:686-701 (finishEmitter)
std::vector<Float3> g_emission;                 // per-triangle emission, src/main.cpp:735-750
std::vector<SpotlightData> g_spots;             // src/main.cpp:883-905
std::vector<float> g_env;                       // RGBA float texels, src/main.cpp:907-930
int g_envW = 0, g_envH = 0;
CameraData g_camera{};                          // src/main.cpp:533-564

std::string resolve(const std::string& scenePath, const std::string& p)
{
    if (p.empty() || p[0] == '/') return p;
    const size_t s = scenePath.find_last_of('/');
    return (s == std::string::npos ? std::string() : scenePath.substr(0, s + 1)) + p;
}

// src/main.cpp:267-401 restated over tinyobjloader and mesh_transform.h
void loadObj(const std::string& path, const TransformDesc& xf, std::vector<TriangleData>& tris)
{
    tinyobj::attrib_t attrib;
    std::vector<tinyobj::shape_t> shapes;
    std::vector<tinyobj::material_t> materials;
    std::string warn, err;
    tinyobj::LoadObj(&attrib, &shapes, &materials, &warn, &err, path.c_str());
    auto V = [&](int i) -> Float3 { return {attrib.vertices[3 * i], attrib.vertices[3 * i + 1], attrib.vertices[3 * i + 2]}; };
    auto N = [&](int i) -> Float3 {
        if (i < 0 || attrib.normals.empty()) return {0, 0, 0};
        return {attrib.normals[3 * i], attrib.normals[3 * i + 1], attrib.normals[3 * i + 2]};
    };
    auto UV = [&](int i) -> Float2 {
        if (i < 0 || attrib.texcoords.empty()) return {0, 0};
        return {attrib.texcoords[2 * i], attrib.texcoords[2 * i + 1]};
    };
    const bool realUV = attrib.texcoords.size() > 2;
    auto planar = [](const Float3& p, const Float3& n) -> Float2 {
        const float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
        if (ay >= ax && ay >= az) return {p.x, p.z};
        if (ax >= ay && ax >= az) return {p.y, p.z};
        return {p.x, p.y};
    };
    for (const auto& sh : shapes) {
        const auto& idx = sh.mesh.indices;
        for (size_t i = 0; i + 2 < idx.size(); i += 3) {
            const auto a = idx[i], b = idx[i + 1], c = idx[i + 2];
            TriangleData t{};
            t.v0 = transformPoint(V(a.vertex_index), xf);
            t.v1 = transformPoint(V(b.vertex_index), xf);
            t.v2 = transformPoint(V(c.vertex_index), xf);
            const bool hasN = a.normal_index >= 0 && b.normal_index >= 0 && c.normal_index >= 0 && !attrib.normals.empty();
            if (hasN) {
                t.n0 = transformNormal(N(a.normal_index), xf);
                t.n1 = transformNormal(N(b.normal_index), xf);
                t.n2 = transformNormal(N(c.normal_index), xf);
            } else {
                const Float3 e1 = {t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z};
                const Float3 e2 = {t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z};
                Float3 g = {e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
                const float len = std::sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
                if (len > 1e-8f) { g.x /= len; g.y /= len; g.z /= len; }
                t.n0 = t.n1 = t.n2 = g;
            }
            if (realUV) { t.uv0 = UV(a.texcoord_index); t.uv1 = UV(b.texcoord_index); t.uv2 = UV(c.texcoord_index); }
            else { t.uv0 = planar(t.v0, t.n0); t.uv1 = planar(t.v1, t.n0); t.uv2 = planar(t.v2, t.n0); }
            tris.push_back(t);
        }
    }
}

float area(const TriangleData& t)
{
    const float ax = t.v1.x - t.v0.x, ay = t.v1.y - t.v0.y, az = t.v1.z - t.v0.z;
    const float bx = t.v2.x - t.v0.x, by = t.v2.y - t.v0.y, bz = t.v2.z - t.v0.z;
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    return 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
}
}  // namespace

// finishEmitter of src/main.cpp:686-701: one EmitterData per emitter whose triangles were just appended
static void finishEmitter(int triIndexOffset, int cdfOffset, float areaSum, const Float3& radiance, float& wsum)
{
    const float lum = 0.2126f * radiance.x + 0.7152f * radiance.y + 0.0722f * radiance.z;
    const float weight = areaSum * lum;
    wsum += weight;
    g_sceneCdf.push_back(wsum);
    EmitterData e{};
    e.triIndexOffset = triIndexOffset;
    e.triCount = (int)g_emTri.size() - triIndexOffset;
    e.cdfOffset = cdfOffset;
    e.radiance = radiance;
    e.areaSum = areaSum;
    e.powerWeight = weight;
    g_emitters.push_back(e);
    ++g_emitterCount;
}

REF_API int refl_load(const char* scenePath)
{
    g_tris.clear(); g_bsdfs.clear(); g_triBsdf.clear(); g_triMat.clear(); g_emTri.clear(); g_emCdf.clear();
    g_sceneCdf.clear(); g_flags.clear(); g_cam.clear();
    g_emitters.clear(); g_emission.clear(); g_spots.clear(); g_env.clear(); g_envW = g_envH = 0;
    const SceneDescription d = loadSceneDescription(scenePath);   // src/scene.cpp:83
    g_matColour.clear(); g_matImage.clear(); g_matW.clear(); g_matH.clear();
    g_matMr.clear(); g_mrW.clear(); g_mrH.clear(); g_emitterCount = 0;
    for (const auto& m : d.materials) {   // src/main.cpp:407-470, :600-612
        float col[3] = {1.0f, 1.0f, 1.0f};
        std::vector<uint8_t> img;
        int w = 1, h = 1, ch = 0;
        if (!m.albedoTexture.empty()) {
            // the path as written, relative to the working directory (main.cpp passes it to stbi_load unchanged)
            unsigned char* px = stbi_load(m.albedoTexture.c_str(), &w, &h, &ch, 4);
            if (px) {
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                const int total = w * h;
                for (int i = 0; i < total; ++i)
                    for (int c = 0; c < 4; ++c) acc[c] += px[4 * i + c] / 255.0;
                for (int c = 0; c < 3; ++c) col[c] = (float)(acc[c] / (double)total);
                img.assign(px, px + (size_t)total * 4);
                stbi_image_free(px);
            } else {
                w = h = 1;
            }
        }
        g_matColour.insert(g_matColour.end(), col, col + 3);
        g_matImage.push_back(img);
        g_matW.push_back(w);
        g_matH.push_back(h);
        g_matMr.emplace_back();
        g_mrW.push_back(1);
        g_mrH.push_back(1);
    }
    for (const auto& b : d.bsdfs) {   // src/main.cpp:629-665
        BsdfData x{};
        if (b.type == "diffuse") { x.type = BSDF_Diffuse; x.p0 = {b.albedoR, b.albedoG, b.albedoB, 0.0f}; }
        else if (b.type == "dielectric") { x.type = BSDF_Dielectric; x.p1 = {b.intIOR, b.extIOR, 0.0f, 0.0f}; }
        else if (b.type == "mirror") {
            x.type = BSDF_Mirror;
            x.p0 = {b.albedoR > 0.0f ? b.albedoR : 1.0f, b.albedoG > 0.0f ? b.albedoG : 1.0f, b.albedoB > 0.0f ? b.albedoB : 1.0f, 0.0f};
        } else if (b.type == "microfacet") {
            x.type = BSDF_Microfacet;
            const float ks = 1.0f - std::fmax(b.albedoR, std::fmax(b.albedoG, b.albedoB));
            x.p0 = {b.albedoR, b.albedoG, b.albedoB, 0.0f};
            x.p1 = {b.alpha, b.intIOR, b.extIOR, ks};
        } else {
            x.type = BSDF_Disney;
            x.p0 = {b.baseColorR, b.baseColorG, b.baseColorB, b.roughness};
            x.p1 = {b.metallic, b.specular, b.specularTransmission, b.specularTint};
            x.p2 = {b.sheen, b.sheenTint, b.subsurface, b.anisotropic};
            x.p3 = {b.clearcoat, b.clearcoatGloss, b.eta, 0.0f};
        }
        g_bsdfs.push_back(x);
    }
    g_sceneCdf.push_back(0.0f);
    float wsum = 0.0f;
    for (const auto& m : d.meshes) {   // src/main.cpp:704-758
        int matId = -1, bsdfId = -1;
        for (size_t i = 0; i < d.materials.size(); ++i) if (d.materials[i].name == m.materialName) matId = (int)i;
        for (size_t i = 0; i < d.bsdfs.size(); ++i) if (d.bsdfs[i].name == d.materials[(size_t)matId].bsdfName) bsdfId = (int)i;
        std::vector<TriangleData> mt;
        loadObj(resolve(scenePath, m.filename), m.transform, mt);
        const Float3 emitColor = {m.radianceR, m.radianceG, m.radianceB};
        const int triIndexOffset = (int)g_emTri.size(), cdfOffset = (int)g_emCdf.size();
        if (m.isEmitter) g_emCdf.push_back(0.0f);
        float a = 0.0f;
        for (const auto& t : mt) {
            g_tris.push_back(t);
            g_triMat.push_back(matId);
            g_triBsdf.push_back(bsdfId);
            g_flags.push_back(m.isEmitter ? 1 : 0);
            g_emission.push_back(m.isEmitter ? emitColor : Float3{0.0f, 0.0f, 0.0f});
            if (m.isEmitter) {
                a += area(t);
                g_emTri.push_back((int)g_tris.size() - 1);
                g_emCdf.push_back(a);
            }
        }
        if (m.isEmitter) finishEmitter(triIndexOffset, cdfOffset, a, emitColor, wsum);
    }
    for (const auto& md : d.models) {   // src/main.cpp:760-817
        const GltfLoadResult gl = loadGltfModel(resolve(scenePath, md.filename), md.transform);
        const int matOffset = (int)g_matW.size(), bsdfOffset = (int)g_bsdfs.size(), firstTri = (int)g_tris.size();
        for (const auto& slot : gl.materials) {
            g_bsdfs.push_back(slot.bsdf);
            const float one[3] = {1.0f, 1.0f, 1.0f};
            g_matColour.insert(g_matColour.end(), one, one + 3);
            g_matImage.push_back(slot.albedo.pixels);
            g_matW.push_back(slot.albedo.width > 0 ? slot.albedo.width : 1);
            g_matH.push_back(slot.albedo.height > 0 ? slot.albedo.height : 1);
            g_matMr.push_back(slot.metallicRoughness.pixels);
            g_mrW.push_back(slot.metallicRoughness.width > 0 ? slot.metallicRoughness.width : 1);
            g_mrH.push_back(slot.metallicRoughness.height > 0 ? slot.metallicRoughness.height : 1);
        }
        for (size_t i = 0; i < gl.triangles.size(); ++i) {
            const int local = gl.materialIds[i];
            const auto& slot = gl.materials[(size_t)local];
            g_tris.push_back(gl.triangles[i]);
            g_triMat.push_back(matOffset + local);
            g_triBsdf.push_back(bsdfOffset + local);
            g_flags.push_back(slot.isEmitter ? 1 : 0);
            g_emission.push_back(slot.isEmitter ? slot.emission : Float3{0.0f, 0.0f, 0.0f});
        }
        for (size_t mi = 0; mi < gl.materials.size(); ++mi) {
            const auto& slot = gl.materials[mi];
            if (!slot.isEmitter) continue;
            const int triIndexOffset = (int)g_emTri.size(), cdfOffset = (int)g_emCdf.size();
            g_emCdf.push_back(0.0f);
            float areaSum = 0.0f;
            const int matId = matOffset + (int)mi;
            for (int ti = firstTri; ti < (int)g_tris.size(); ++ti) {
                if (g_triMat[(size_t)ti] != matId) continue;
                areaSum += area(g_tris[(size_t)ti]);
                g_emTri.push_back(ti);
                g_emCdf.push_back(areaSum);
            }
            if (areaSum > 0.0f) finishEmitter(triIndexOffset, cdfOffset, areaSum, slot.emission, wsum);
        }
    }
    for (const auto& sd : d.spotlights) {   // src/main.cpp:883-905
        SpotlightData sp{};
        sp.position = {sd.posX, sd.posY, sd.posZ};
        float dx = sd.dirX, dy = sd.dirY, dz = sd.dirZ;
        const float dlen = sqrtf(dx * dx + dy * dy + dz * dz);
        if (dlen > 1e-6f) { dx /= dlen; dy /= dlen; dz /= dlen; }
        sp.direction = {dx, dy, dz};
        sp.radiance = {sd.radianceR, sd.radianceG, sd.radianceB};
        sp.intensity = sd.intensity;
        const float kPi = 3.14159265358979323846f;
        sp.innerConeCosine = cosf(sd.innerConeAngle * kPi / 180.0f);
        sp.outerConeCosine = cosf(sd.outerConeAngle * kPi / 180.0f);
        g_spots.push_back(sp);
    }
    if (!d.envMapPath.empty()) {   // src/main.cpp:907-930 (path taken relative to the scene file, as the OBJs)
        int comp = 0;
        float* rgb = stbi_loadf(resolve(scenePath, d.envMapPath).c_str(), &g_envW, &g_envH, &comp, 3);
        if (!rgb) return -1;
        g_env.assign((size_t)g_envW * g_envH * 4, 1.0f);
        for (size_t i = 0; i < (size_t)g_envW * g_envH; ++i)
            for (int c = 0; c < 3; ++c) g_env[4 * i + c] = rgb[3 * i + c];
        stbi_image_free(rgb);
    }
    {   // src/main.cpp:533-564, with GLM's normalize (v * 1/sqrt(dot)), cross and radians
        const CameraDesc& c = d.camera;
        const Float3 eye = {c.eyeX, c.eyeY, c.eyeZ}, up = {c.upX, c.upY, c.upZ};
        const Float3 tgt = {c.lookAtX, c.lookAtY, c.lookAtZ};
        auto cross = [](Float3 x, Float3 y) {
            return Float3{x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
        };
        auto normalize = [](Float3 v) {
            const float inv = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
            return Float3{v.x * inv, v.y * inv, v.z * inv};
        };
        const Float3 forward = normalize(Float3{tgt.x - eye.x, tgt.y - eye.y, tgt.z - eye.z});
        const Float3 right = normalize(cross(forward, up));
        g_camera.origin = eye;
        g_camera.forward = forward;
        g_camera.right = right;
        g_camera.up = cross(right, forward);
        g_camera.fovYRadians = c.fovYDegrees * 0.01745329251994329576923690768489f;
        g_camera.aspect = (float)d.windowWidth / (float)d.windowHeight;
    }
    const CameraDesc& c = d.camera;
    g_cam = {c.eyeX, c.eyeY, c.eyeZ, c.lookAtX, c.lookAtY, c.lookAtZ, c.upX, c.upY, c.upZ, c.fovYDegrees,
             (float)d.windowWidth, (float)d.windowHeight, d.envMapIntensity, d.envMapRotation, (float)d.spotlights.size()};
    return (int)g_tris.size();
}

REF_API int refl_material_count(void) { return (int)g_matW.size(); }
REF_API int refl_emitter_count(void) { return g_emitterCount; }

// metallic-roughness image of material i: sizes; returns 1 when present (copied to `rgba` when non-null)
REF_API int refl_material_mr(int i, int* w, int* h, uint8_t* rgba)
{
    *w = g_mrW[(size_t)i];
    *h = g_mrH[(size_t)i];
    if (g_matMr[(size_t)i].empty()) return 0;
    if (rgba) std::memcpy(rgba, g_matMr[(size_t)i].data(), g_matMr[(size_t)i].size());
    return 1;
}

// colour[3], image size; returns 1 when the material has an image (copied to `rgba` when non-null)
REF_API int refl_material(int i, float* colour, int* w, int* h, uint8_t* rgba)
{
    std::memcpy(colour, &g_matColour[3 * (size_t)i], 3 * sizeof(float));
    *w = g_matW[(size_t)i];
    *h = g_matH[(size_t)i];
    if (g_matImage[(size_t)i].empty()) return 0;
    if (rgba) std::memcpy(rgba, g_matImage[(size_t)i].data(), g_matImage[(size_t)i].size());
    return 1;
}

REF_API int refl_counts(int* out)
{
    out[0] = (int)g_tris.size(); out[1] = (int)g_bsdfs.size(); out[2] = (int)g_emTri.size();
    out[3] = (int)g_emCdf.size(); out[4] = (int)g_sceneCdf.size(); out[5] = (int)g_cam.size();
    return 0;
}

REF_API void refl_copy(TriangleData* tris, BsdfData* bsdfs, int* triBsdf, int* triMat, uint8_t* flags, int* emTri,
                       float* emCdf, float* sceneCdf, float* cam)
{
    std::memcpy(tris, g_tris.data(), g_tris.size() * sizeof(TriangleData));
    std::memcpy(bsdfs, g_bsdfs.data(), g_bsdfs.size() * sizeof(BsdfData));
    std::memcpy(triBsdf, g_triBsdf.data(), g_triBsdf.size() * sizeof(int));
    std::memcpy(triMat, g_triMat.data(), g_triMat.size() * sizeof(int));
    std::memcpy(flags, g_flags.data(), g_flags.size());
    std::memcpy(emTri, g_emTri.data(), g_emTri.size() * sizeof(int));
    std::memcpy(emCdf, g_emCdf.data(), g_emCdf.size() * sizeof(float));
    std::memcpy(sceneCdf, g_sceneCdf.data(), g_sceneCdf.size() * sizeof(float));
    std::memcpy(cam, g_cam.data(), g_cam.size() * sizeof(float));
}

// The rest of what src/main.cpp:836-930 uploads: emitter table, per-triangle emission, spotlights, the env map
// (RGBA float) and the camera.  Sizes first (null pointers), then copies.
REF_API int refl_extras_counts(int* out)
{
    out[0] = (int)g_emitters.size(); out[1] = (int)g_emission.size(); out[2] = (int)g_spots.size();
    out[3] = g_envW; out[4] = g_envH;
    return 0;
}

REF_API void refl_extras_copy(EmitterData* emitters, Float3* emission, SpotlightData* spots, float* envRGBA,
                              CameraData* camera)
{
    if (!g_emitters.empty()) std::memcpy(emitters, g_emitters.data(), g_emitters.size() * sizeof(EmitterData));
    if (!g_emission.empty()) std::memcpy(emission, g_emission.data(), g_emission.size() * sizeof(Float3));
    if (!g_spots.empty()) std::memcpy(spots, g_spots.data(), g_spots.size() * sizeof(SpotlightData));
    if (!g_env.empty()) std::memcpy(envRGBA, g_env.data(), g_env.size() * sizeof(float));
    std::memcpy(camera, &g_camera, sizeof(CameraData));
}
