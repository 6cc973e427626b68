// bte_compat.cpp -- reference-named C++ entry points (bte/render_kernel.h) over the
// C-ABI.  Errors terminate the process, as the reference's CUDA_CHECK does.
#include "../../include/bte/render_kernel.h"

#include <cstdio>
#include <cstdlib>

namespace {
void die(const char* fn)
{
    std::fprintf(stderr, "[bte] %s failed: %s\n", fn, bte_last_error());
    std::exit(EXIT_FAILURE);
}
inline void ok(int rc, const char* fn) { if (rc < 0) die(fn); }
}  // namespace

void cudaInitOptix() { ok(bte_init_accel(), "cudaInitOptix"); }
void cudaInitScene(const TriangleData* t, int n, const Float3* m, int mc, const int* ids, int w, int h)
{
    ok(bte_init_scene(t, n, m, mc, ids, w, h), "cudaInitScene");
}
void cudaInit(const TriangleData& tri, const Float3& color, int w, int h) { ok(bte_init(&tri, &color, w, h), "cudaInit"); }
void cudaInitCamera(const CameraData& camera) { ok(bte_init_camera(&camera), "cudaInitCamera"); }
void cudaInitTriangleEmission(const Float3* e, int n) { ok(bte_init_triangle_emission(e, n), "cudaInitTriangleEmission"); }
void cudaInitTriangleEmitterFlags(const uint8_t* f, int n)
{
    ok(bte_init_triangle_emitter_flags(f, n), "cudaInitTriangleEmitterFlags");
}
void cudaInitEmitterTable(const EmitterData* e, int ec, const int* ti, int tic, const float* tcdf, int tcc, const float* scdf)
{
    ok(bte_init_emitter_table(e, ec, ti, tic, tcdf, tcc, scdf), "cudaInitEmitterTable");
}
void cudaInitBsdfs(const BsdfData* b, int bc, const int* ids, int n) { ok(bte_init_bsdfs(b, bc, ids, n), "cudaInitBsdfs"); }
void cudaInitSpotlights(const SpotlightData* s, int n) { ok(bte_init_spotlights(s, n), "cudaInitSpotlights"); }
void cudaInitTextures(const uint8_t* const* p, const int* w, const int* h, int n)
{
    ok(bte_init_textures(p, w, h, n), "cudaInitTextures");
}
void cudaInitMrTextures(const uint8_t* const* p, const int* w, const int* h, int n)
{
    ok(bte_init_mr_textures(p, w, h, n), "cudaInitMrTextures");
}
void cudaInitEnvMap(const float* rgba, int w, int h, float intensity, float rot)
{
    ok(bte_init_env_map(rgba, w, h, intensity, rot), "cudaInitEnvMap");
}
void cudaRegisterPBO(uint32_t)
{
    std::fprintf(stderr, "[bte] cudaRegisterPBO: no OpenGL on this build; use cudaSetOutputBuffer or bte_read_framebuffer\n");
    std::exit(EXIT_FAILURE);
}
void cudaSetOutputBuffer(uint32_t* dev) { ok(bte_set_output_buffer(dev), "cudaSetOutputBuffer"); }
void cudaResetAccumulation(int w, int h) { ok(bte_reset_accumulation(w, h), "cudaResetAccumulation"); }
void cudaRender(int w, int h) { ok(bte_render(w, h), "cudaRender"); }
bool cudaToggleDenoiser()
{
    const int r = bte_toggle_denoiser();
    if (r < 0) die("cudaToggleDenoiser");
    return r != 0;
}
void cudaSetRenderMode(RenderMode mode)
{
    ok(bte_set_render_mode(mode == RenderMode::Wavefront ? BTE_RENDER_WAVEFRONT : BTE_RENDER_MEGAKERNEL), "cudaSetRenderMode");
}
RenderMode cudaGetRenderMode()
{
    return bte_get_render_mode() == BTE_RENDER_WAVEFRONT ? RenderMode::Wavefront : RenderMode::Megakernel;
}
void cudaCleanup() { ok(bte_cleanup(), "cudaCleanup"); }
