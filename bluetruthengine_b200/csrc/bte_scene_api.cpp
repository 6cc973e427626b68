// bte_scene_api.cpp -- C-ABI over the scene loader (host only; needs no GPU
// except for bte_scene_upload).
#include "bte_internal.h"

#include <new>

struct BteScene {
    bte::SceneData data;
    std::vector<const uint8_t*> albedoPtrs, mrPtrs;
};

extern "C" {

int bte_scene_load(const char* scenePath, BteScene** out)
{
    if (!out) { bte::setError("bte_scene_load: null output pointer"); return -1; }
    *out = nullptr;
    BteScene* s = new (std::nothrow) BteScene();
    if (!s) { bte::setError("bte_scene_load: out of memory"); return -1; }
    std::string err;
    if (bte::sceneLoad(scenePath, s->data, err) != 0) {
        delete s;
        bte::setError("bte_scene_load: " + err);
        return -1;
    }
    *out = s;
    return 0;
}

int bte_scene_arrays(const BteScene* scene, BteSceneArrays* o)
{
    if (!scene || !o) { bte::setError("bte_scene_arrays: null argument"); return -1; }
    const bte::SceneData& d = scene->data;
    *o = BteSceneArrays{};
    o->triangles = d.triangles.data(); o->triangleCount = static_cast<int>(d.triangles.size());
    o->materials = d.materials.data(); o->materialCount = static_cast<int>(d.materials.size());
    o->triangleMaterialIds = d.triangleMaterialIds.data();
    o->triangleBsdfIds = d.triangleBsdfIds.data();
    o->bsdfs = d.bsdfs.data(); o->bsdfCount = static_cast<int>(d.bsdfs.size());
    o->triangleEmission = d.triangleEmission.data();
    o->triangleEmitterFlags = d.triangleEmitterFlags.data();
    o->emitters = d.emitters.data(); o->emitterCount = static_cast<int>(d.emitters.size());
    o->emitterTriIndices = d.emitterTriIndices.data(); o->emitterTriIndexCount = static_cast<int>(d.emitterTriIndices.size());
    o->emitterTriCdf = d.emitterTriCdf.data(); o->emitterTriCdfCount = static_cast<int>(d.emitterTriCdf.size());
    o->sceneEmitterCdf = d.sceneEmitterCdf.data();
    o->spotlights = d.spotlights.data(); o->spotlightCount = static_cast<int>(d.spotlights.size());
    o->envRGBA = d.envRGBA.empty() ? nullptr : d.envRGBA.data();
    o->envWidth = d.envWidth; o->envHeight = d.envHeight;
    o->envIntensity = d.envIntensity; o->envRotationDeg = d.envRotationDeg;
    o->camera = d.camera;
    o->width = d.width; o->height = d.height;
    BteScene* s = const_cast<BteScene*>(scene);
    s->albedoPtrs.clear();
    s->mrPtrs.clear();
    for (const auto& im : d.albedoImages) s->albedoPtrs.push_back(im.empty() ? nullptr : im.data());
    for (const auto& im : d.mrImages) s->mrPtrs.push_back(im.empty() ? nullptr : im.data());
    o->albedoPixels = s->albedoPtrs.empty() ? nullptr : s->albedoPtrs.data();
    o->albedoWidths = d.albedoWidths.data(); o->albedoHeights = d.albedoHeights.data();
    o->mrPixels = s->mrPtrs.empty() ? nullptr : s->mrPtrs.data();
    o->mrWidths = d.mrWidths.data(); o->mrHeights = d.mrHeights.data();
    return 0;
}

void bte_scene_free(BteScene* scene) { delete scene; }

// The upload order of src/main.cpp:819-930.
int bte_scene_upload(const BteScene* scene)
{
    if (!scene) { bte::setError("bte_scene_upload: null scene"); return -1; }
    const bte::SceneData& d = scene->data;
    const int T = static_cast<int>(d.triangles.size());
    int rc = bte_init_camera(&d.camera);
    {   // uploadLayer, src/main.cpp:819-838: one entry per material, NULL where it has no image
        std::vector<const uint8_t*> a, m;
        for (const auto& im : d.albedoImages) a.push_back(im.empty() ? nullptr : im.data());
        for (const auto& im : d.mrImages) m.push_back(im.empty() ? nullptr : im.data());
        if (rc == 0) rc = bte_init_textures(a.empty() ? nullptr : a.data(), d.albedoWidths.data(), d.albedoHeights.data(),
                                            static_cast<int>(a.size()));
        if (rc == 0) rc = bte_init_mr_textures(m.empty() ? nullptr : m.data(), d.mrWidths.data(), d.mrHeights.data(),
                                               static_cast<int>(m.size()));
    }
    if (rc == 0) rc = bte_init_scene(d.triangles.data(), T, d.materials.data(), static_cast<int>(d.materials.size()),
                                     d.triangleMaterialIds.data(), d.width, d.height);
    if (rc == 0) rc = bte_init_accel();
    if (rc == 0) rc = bte_init_triangle_emission(d.triangleEmission.data(), T);
    if (rc == 0) rc = bte_init_triangle_emitter_flags(d.triangleEmitterFlags.data(), T);
    if (rc == 0) {
        if (!d.emitters.empty())
            rc = bte_init_emitter_table(d.emitters.data(), static_cast<int>(d.emitters.size()), d.emitterTriIndices.data(),
                                        static_cast<int>(d.emitterTriIndices.size()), d.emitterTriCdf.data(),
                                        static_cast<int>(d.emitterTriCdf.size()), d.sceneEmitterCdf.data());
        else
            rc = bte_init_emitter_table(nullptr, 0, nullptr, 0, nullptr, 0, nullptr);
    }
    if (rc == 0) rc = bte_init_bsdfs(d.bsdfs.data(), static_cast<int>(d.bsdfs.size()), d.triangleBsdfIds.data(), T);
    if (rc == 0) rc = bte_init_spotlights(d.spotlights.empty() ? nullptr : d.spotlights.data(),
                                          static_cast<int>(d.spotlights.size()));
    if (rc == 0) rc = bte_init_env_map(d.envRGBA.empty() ? nullptr : d.envRGBA.data(), d.envWidth, d.envHeight,
                                       d.envIntensity, d.envRotationDeg);
    return rc;
}

}  // extern "C"
