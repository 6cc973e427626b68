/*
 * bte/render_api.h -- C-ABI of the B200 wavefront path tracer (libbte_b200.so).
 *
 * Drop-in boundary for Blue Truth Engine's renderer API.  Every entry point
 * replaces one free function of the reference's include/render_kernel.h (cited
 * per function, paths relative to the reference project root) with an
 * extern "C" twin that takes plain pointers and sizes and returns a status
 * (0 = success, negative = error; bte_last_error() describes the last error
 * of the calling thread).  The reference aborts the process on any error
 * (src/host/cuda_check.h:14-32); the reference-named C++ wrappers in
 * bte/render_kernel.h keep that behaviour for drop-in callers.
 *
 * POD types are byte-identical to render_kernel.h:9-94.  Inputs are
 * caller-owned host arrays copied synchronously during the call; the library
 * owns the device copies; re-calling replaces; NULL/0 clears (as
 * src/host/scene_upload.cu:18-198).  Not re-entrant: one renderer state per
 * process, driven from one thread, like the reference's globals.
 */
#ifndef BTE_RENDER_API_H
#define BTE_RENDER_API_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- POD types: render_kernel.h:9-94 ---- */
typedef struct { float x, y; } Float2;
typedef struct { float x, y, z; } Float3;
typedef struct { float x, y, z, w; } Float4;
typedef struct { Float3 v0, v1, v2; Float3 n0, n1, n2; Float2 uv0, uv1, uv2; } TriangleData;      /* 96 B */
typedef struct { Float3 origin, forward, right, up; float fovYRadians, aspect; } CameraData;       /* 56 B */
typedef struct { int triIndexOffset, triCount, cdfOffset; Float3 radiance; float areaSum, powerWeight; } EmitterData;
typedef struct { Float3 position, direction, radiance; float intensity, innerConeCosine, outerConeCosine; } SpotlightData;
typedef struct { int type; Float4 p0, p1, p2, p3; } BsdfData;                                      /* 68 B */
enum { BSDF_Diffuse = 1, BSDF_Dielectric = 2, BSDF_Mirror = 3, BSDF_Microfacet = 4, BSDF_Disney = 5 };

/* render_kernel.h:199-202.  Wavefront: the staged path tracer.  Megakernel: the reference's megakernel
 * (src/optix_programs.cu:54-108): one thread and one RNG stream per pixel through 5 paths, one Welford update
 * per frame; bte_read_accum_f64 then holds a sum of per-frame means (divide by the frame count, which
 * bte_get_frame_index reports in this mode). */
enum { BTE_RENDER_MEGAKERNEL = 0, BTE_RENDER_WAVEFRONT = 1 };

/* env-map importance sampling: the reference's marginal/conditional CDF
 * (rt_env_map.cuh:82-199, bit-exact) or FP64-built two-level alias tables. */
enum { BTE_ENV_SAMPLING_CDF = 0, BTE_ENV_SAMPLING_ALIAS = 1 };

/* Runtime knobs that are compile-time constants in the reference
 * (include/rt_constants.cuh:11-19, rt_path_integrator.cuh:56). */
typedef struct {
    int samplesPerFrame;   /* paths per pixel per bte_render call (reference wavefront: 1) */
    int maxDepth;          /* extend+shade steps per path (reference: MAX_BOUNCES = 200) */
    int rrStart;           /* roulette when bounceCount > rrStart (reference: 3) */
    int envSampling;       /* BTE_ENV_SAMPLING_* */
    int blockSize;         /* threads per block of the stage kernels (0 = default) */
    int useGraph;          /* capture the frame's launch sequence in a CUDA graph */
} BteRenderConfig;

typedef struct {
    int64_t samples;       /* camera paths traced by the last bte_render */
    int64_t extends;       /* closest-hit rays (path segments) */
    int64_t shadowRays;    /* NEE shadow rays */
    int maxBounceReached;  /* deepest bounce with a non-empty queue */
    float msTotal;         /* device time of the last frame (CUDA events) */
    float msGenerate, msExtend, msShade, msConnect, msPresent;  /* per stage (only with timing enabled) */
    float msTail;          /* the tail kernel (BteTuning.tailPaths), timing enabled */
    int tailBounce;        /* first bounce finished by the tail kernel, or -1 */
    int64_t tailExtends;   /* closest-hit rays traced by the tail kernel (included in extends) */
    int64_t tailShadowRays;/* shadow rays traced by the tail kernel (included in shadowRays) */
} BteFrameStats;

const char* bte_last_error(void);
int bte_version(void);

/* ---- scene uploads: render_kernel.h:100-174 ---- */
int bte_init_scene(const TriangleData* triangles, int triangleCount, const Float3* materials, int materialCount,
                   const int* triangleMaterialIds, int imageWidth, int imageHeight);       /* cudaInitScene :111 */
int bte_init(const TriangleData* tri, const Float3* color, int imageWidth, int imageHeight); /* cudaInit :117 */
int bte_init_accel(void);                                   /* cudaInitOptix :103 -> LBVH build */
int bte_init_camera(const CameraData* camera);              /* cudaInitCamera :121 */
int bte_init_triangle_emission(const Float3* emission, int triangleCount);      /* :125 */
int bte_init_triangle_emitter_flags(const uint8_t* flags, int triangleCount);   /* :129 */
int bte_init_emitter_table(const EmitterData* emitters, int emitterCount, const int* emitterTriIndices,
                           int emitterTriIndexCount, const float* emitterTriCdf, int emitterTriCdfCount,
                           const float* sceneEmitterCdf);                        /* :137 */
int bte_init_bsdfs(const BsdfData* bsdfs, int bsdfCount, const int* triangleBsdfIds, int triangleCount); /* :143 */
int bte_init_spotlights(const SpotlightData* spotlights, int spotlightCount);  /* :148 */
int bte_init_textures(const uint8_t* const* pixels, const int* widths, const int* heights, int count);    /* :155 */
int bte_init_mr_textures(const uint8_t* const* pixels, const int* widths, const int* heights, int count); /* :163 */
int bte_init_env_map(const float* rgba, int width, int height, float intensity, float rotationDeg);      /* :173 */

/* ---- frame API: render_kernel.h:177-211 ---- */
int bte_set_output_buffer(uint32_t* deviceRGBA8);   /* replaces cudaRegisterPBO :177 (no GL on the box) */
int bte_reset_accumulation(int imageWidth, int imageHeight);                    /* :183 */
int bte_render(int imageWidth, int imageHeight);                                /* :187 */
/* Batched views (no reference counterpart; the reference renders one camera per cudaRender): several
 * camera views of the current scene, each of its own size and samples per frame, rendered in one launch
 * sequence over their concatenated paths.  View slot i keeps its own accumulation across calls (a changed
 * size restarts it); the per-view images equal those of bte_render with that camera, bit for bit. */
typedef struct {
    CameraData camera;
    int width, height;
    int samplesPerFrame;   /* 0: the view is idle this frame (its accumulation is kept); not all views may be 0 */
} BteView;
int bte_render_views(const BteView* views, int count);            /* at most 64 views */
int bte_read_view_accum(int view, float* hostRGB, double* hostRGBSum);   /* W*H*3 each; either may be NULL */
int bte_reset_views(void);
/* Scene slots (no reference counterpart; the reference holds one scene): up to 8 independent scenes, each
 * with its own geometry, tree, materials, lights, env map, configuration, streams and view accumulations.
 * Every upload, configuration and render call acts on the selected slot (slot 0 at start). */
int bte_select_scene(int scene);                    /* 0..7 */
int bte_get_selected_scene(int* scene);
/* Several scenes' view batches in one call: scene scenes[i] renders the next viewCounts[i] entries of views.
 * Every scene's launch sequence is enqueued on its own streams before any host wait, so the scenes run side by
 * side on the GPU; each scene's views accumulate exactly as bte_render_views on that slot would leave them.
 * Slots must be distinct; the selected slot is unchanged afterwards. */
int bte_render_scene_batch(const int* scenes, const int* viewCounts, const BteView* views, int sceneCount);
/* How bte_render_scene_batch runs the scenes.  1 (the default): every view of every scene in ONE launch sequence
 * (one generate, one extend / shade / connect per bounce, one present over all scenes' paths), each path looking
 * its scene -- geometry, tree, materials, lights, env map -- up in a per-frame scene table; this needs every scene
 * in wavefront mode with the 8-wide tree and the first scene's max depth, roulette start, block size and graph
 * use, and the frame-level tuning is the first scene's; other batches fall back to mode 0.  0: each scene's own
 * launch sequence, the scenes side by side on their own streams (one parent graph when all use graphs).  Frame
 * stats of every scene in a one-sequence batch are the batch's, with each scene's own sample count. */
int bte_set_batch_mode(int mode);
int bte_get_batch_mode(int* mode);
int bte_toggle_denoiser(void);                      /* :192; returns new state (0/1) or <0; needs denoiser weights */
int bte_read_denoised(float* hostRGB);               /* W*H*3 denoised mean radiance of the last frame (denoiser on) */
int bte_set_render_mode(int mode);                                              /* :205 */
int bte_get_render_mode(void);                                                  /* :208 */
int bte_cleanup(void);                                                          /* :211 */

/* ---- additions (no reference counterpart; headless replacements of the PBO path) ---- */
int bte_set_render_config(const BteRenderConfig* cfg);
int bte_get_render_config(BteRenderConfig* cfg);
int bte_get_frame_stats(BteFrameStats* out);
int bte_set_stage_timing(int enabled);
int bte_get_frame_index(uint32_t* out);              /* samples accumulated so far */
int bte_set_frame_index(uint32_t frameIndex);        /* resume an accumulation at a sample index */
int bte_read_framebuffer(uint32_t* hostRGBA8);       /* W*H packed ABGR, rt_path_integrator.cuh:93-105 */
int bte_read_accum(float* hostRGB);                  /* FP32 Welford mean, W*H*3 */
int bte_read_accum_f64(double* hostRGBSum);          /* FP64 running sum of samples, W*H*3 */
int bte_read_sample_radiance(float* hostRGB, int count);  /* per-path radiance of the last frame [W*H*spp*3] */
int bte_read_hit_log(int* hostTri, int count);       /* per-bounce closest-hit triangle of the last frame */
int bte_set_hit_log(int enabled);                    /* record [path][bounce] hit triangles (debug/parity) */
/* Denoiser features: per-pixel running means of the material colour (BsdfData
 * p0.xyz after textures) and shading normal at each path's first hit that is
 * not a perfect mirror or dielectric, seen through the mirrors and dielectrics
 * in front of it (colour times their tints: a mirror's p0.xyz, 1 for a
 * dielectric; a path that meets only such surfaces keeps the last one's normal
 * and the product so far; 0 when the first ray misses), accumulated with the
 * radiance.  Read as [W*H][albedo.xyz, normal.xyz]. */
int bte_set_aov(int enabled);
int bte_read_aov(float* hostAlbedoNormal);
/* Acceleration-structure and kernel tuning (what the autotuner sweeps).
 * Width and leaf size apply at the next bte_init_accel, the rest at once. */
typedef struct {
    int bvhWidth;          /* 2: binary LBVH; 8: 8-wide tree with 8-bit quantised child boxes */
    int maxLeafTriangles;  /* 1-64 (binary tree), 1-3 (8-wide tree) */
    int shadeMinBlocks;    /* register budget of the shade kernel: 2, 3 or 4 resident blocks of 256 threads per
                            * SM (96, 72 or 64 registers per thread; 5, 7 or 8 blocks of 128 threads) */
    int postponePercent;   /* 8-wide walk: a lane defers its leaf tests while fewer than this
                            * percentage of the warp's lanes have leaf tests (0 = never, 0-100) */
    int sortShading;       /* 1: extend buckets paths by hit material (miss, BSDF type) and shade runs the
                            * buckets in order; 0: shade runs the extend queue as it is */
    int tailPaths;         /* from the first bounce whose queue is shorter than this, one kernel finishes the
                            * remaining paths (extend + shade + shadow rays per bounce, each path's bounces back
                            * to back; eight lanes walk a path's rays over the 8-wide tree, one thread per path
                            * over the binary tree); 0: the wavefront runs every bounce (default 4096) */
    int bvhBuilder;        /* binary hierarchy the trees are built from: 0 Morton-prefix splits (Karras 2012);
                            * 1 PLOC, locally-ordered clustering over the Morton order (Meister & Bittner 2018) */
    int plocRadius;        /* PLOC neighbour search radius in positions, 1-32 */
    int overlapConnect;    /* 1: bounce b's shadow rays run on a second stream beside bounce b+1's closest-hit
                            * rays (they share no data); 0: the stages run one after another */
    int wideCollapse;      /* children of each 8-wide node: 0 greedy (open the largest-area child first);
                            * 1 surface-area-optimal (dynamic program of Ylitie, Karras & Laine 2017) */
    int raySortBits;       /* 0: off; 1-4: before the closest-hit rays of bounces 1..raySortBounces (queues of at
                            * least 32768 rays), the queue is reordered by direction octant and origin cell
                            * (raySortBits bits per axis of the scene's bounding cube), so a warp traces nearby
                            * rays of one octant; results do not depend on it */
    int raySortBounces;    /* last bounce reordered, 1-64 */
    int leafTestsPerStep;  /* 8-wide walk: 0 tests all triangles of a node's hit leaves in the step that fetched
                            * the node; 1-24 tests at most that many per step and fetches the next node only
                            * when they are done (lanes with many triangles hold their warp less long) */
    int orderBounces;      /* 0: off; 1-64: for bounces 0..orderBounces-1 the material buckets and the next
                            * bounce's queue are rebuilt in ascending path order by a stable compaction over
                            * path indices (instead of atomic appends in completion order), so a warp's paths
                            * are neighbours in the path-state arrays (default 3); active only with
                            * sortShading 1 and raySortBits 0; results do not depend on it */
} BteTuning;
int bte_set_tuning(const BteTuning* tuning);
int bte_get_tuning(BteTuning* tuning);
/* The acceleration structure in use: width (2 or 8), node count, levels of
 * the 8-wide tree (0 for width 2) and device build time. */
int bte_get_accel_info(int* width, int* nodeCount, int* depth, float* msBuild);
/* The binary hierarchy the structure in use was built from (BteTuning.bvhBuilder; a
 * PLOC tree too deep for the binary walk's stack is rebuilt with Morton-prefix splits). */
int bte_get_accel_builder(int* builder);

/* ---- learned denoiser (replaces the vendor denoiser stage, render_kernel.h:187 / src/host/denoiser.cu) ----
 * A 5-level U-Net (3x3 convolutions, 32-128 channels) over log(1 + radiance)
 * plus the feature albedo and normal (bte_set_aov), BF16 tensor-core convolutions with FP32
 * accumulation, FP32 master weights trained with Adam on L1 in log space.
 * Images are row-major [H][W][3] radiance and [H][W][6] features (albedo xyz,
 * normal xyz, as bte_read_aov returns them). */
int bte_denoiser_init(uint64_t seed);                            /* random (He) initialisation */
int bte_denoiser_param_count(long long* count);
int bte_denoiser_get_params(float* hostParams, long long count);
int bte_denoiser_set_params(const float* hostParams, long long count);
int bte_denoiser_set_dataset(const float* noisy, const float* features, const float* target, int count, int width,
                             int height);                        /* training images, copied to the device */
int bte_denoiser_train(int steps, int batch, int crop, float learningRate, uint64_t seed, float* lossPerStep);
int bte_denoiser_denoise(const float* radiance, const float* features, int width, int height, float* out);
int bte_denoiser_last_ms(float* ms);                             /* device time of the last denoise / train call */
/* The tensor-core kernels' bounded pipeline wait on a barrier that nothing completes: *status 2 when the wait
 * gave up as designed (after about two seconds; the context stays usable), 1 if it returned as completed;
 * *seconds its duration.  A check of the failure path without a fault. */
int bte_denoiser_debug_wait_timeout(unsigned int* status, double* seconds);
int bte_denoiser_set_tcgen05(int mode);   /* conv kernels: 0 warp-level MMA, 1 tcgen05 pixel tiles, 2 row tiles (default), 3 row tiles upsampling in-kernel */
/* Weight gradients of training: 1 (default) the tcgen05 kernel (pixels as the reduction axis over channel-major
 * copies) for layers whose image width is a multiple of 8 and pixel count a multiple of 64, the warp-level kernel
 * for the rest; 0 the warp-level mma.sync kernel for every layer; 2-7 the tcgen05 kernel with one of its pipeline
 * shapes (stages, copy lag, pixels per stage): 2 (3, 2, 64), 3 (4, 2, 64), 4 (6, 4, 32), 5 (5, 3, 32) with
 * zero-filling copies, 6 (3, 2, 64) and 7 (5, 3, 32) with plain copies and shared-memory zero stores; a tuning
 * choice with the same sums. */
int bte_denoiser_set_wgrad(int kind);
int bte_denoiser_debug_conv(int op, const float* x, const float* w, const float* bias, const float* dy, int n, int h,
                            int w_, int cin, int cout, int relu, float* out);

/* ---- debug/parity entry points over device-resident state ---- */
/* The LBVH's integer steps for n host triangles (the acceleration-structure build replacing
 * src/host/optix_setup.cu:215-292): the 63-bit Morton code of each triangle's centroid (21 bits per axis
 * over the centroid bounds, x in the highest interleaved bit) and the triangle order after the stable
 * radix sort by code (ties in ascending index). */
int bte_debug_lbvh_order(const TriangleData* triangles, int n, uint64_t* mortonKeys, int* sortedOrder);
/* closest hit for n rays [origin, dir] (host arrays): triangle index (-1 miss) and t, u, v */
int bte_trace_closest(const float* rays, int n, int* outTri, float* outTuv);
int bte_trace_occluded(const float* rays, const float* tmax, int n, uint8_t* outOccluded);
/* The same with the walk chosen: lanesPerRay 1 (one lane per ray, the walk of the bulk of a frame) or
 * 8 (eight lanes per ray, the walk of the last bounces; needs the 8-wide tree).  Same results. */
int bte_trace_closest_lanes(const float* rays, int n, int lanesPerRay, int* outTri, float* outTuv);
int bte_trace_occluded_lanes(const float* rays, const float* tmax, int n, int lanesPerRay, uint8_t* outOccluded);
/* env-map queries through the device tables */
int bte_env_query(int op, const float* in, int n, float* out);   /* op 0 eval, 1 pdf, 2 sample */
int bte_env_tables(float* marginal, float* conditional, float* totalPower);      /* CDF mode tables */
int bte_env_alias_tables(float* rowProb, int* rowIdx, float* colProb, int* colIdx, float* pixelPdf);
/* deterministic elementary functions as evaluated on the device */
int bte_math_eval(int fn, const float* a, const float* b, float* out, int n);
/* BSDF queries evaluated on the device */
int bte_bsdf_query(const BsdfData* bsdf, int op, const float* wi, const float* woOrU, int n, float* out);
/* hardware texture fetch vs the library's software filter, for the texture-filter pin */
int bte_tex_hw_vs_sw(const float* texels, int w, int h, int wrapV, const float* uv, int n, float* outHw, float* outSw);

/* ---- env-map alias tables without allocation ----
 * No counterpart in the reference.  Builds the same FP64 alias tables and
 * per-pixel pdf that bte_init_env_map builds, for a caller that cannot
 * allocate device memory at that point (cudaMalloc/cudaFree synchronise the
 * whole device; some hosts reserve all device memory for their own pool).
 * Inputs and outputs are the caller's device buffers: dTexelsRGBA is
 * width*height float4 texels (16-byte aligned), outputs are rowProb/rowAlias
 * [height], colProb/colAlias/pixelPdf [width*height] and the FP64 total
 * weight [1].  Work is queued on `stream` (0 = default stream) and nothing is
 * allocated: the intermediates live in one fixed device array, so maps are
 * limited to 131072 texels (e.g. 512x256) and 4096 rows; larger sizes return
 * an error.  The array's device address is looked up once per device, by the
 * renderer's device set-up (any renderer call) or else by the first call here;
 * under lazy module loading that is also when the array's memory is taken, so
 * make one of those calls before reserving the rest of device memory, and the
 * first call here before any stream capture.  dTotalPower must be 8-byte
 * aligned.  All calls share the array: calls whose kernels overlap on the GPU
 * race and must be serialised by the caller. */
int bte_env_build_alias_noalloc(const float* dTexelsRGBA, int width, int height, float* dRowProb, int* dRowAlias,
                                float* dColProb, int* dColAlias, float* dPixelPdf, double* dTotalPower, void* stream);

/* ---- headless output (replaces the window of src/main.cpp: screenshots :118-142, recording :72-116 and
 * :990-997, the scene-changed reset of :947-952) ---- */
int bte_get_framebuffer_size(int* width, int* height);   /* of the last frame's packed RGBA8 framebuffer */
int bte_mark_scene_changed(void);    /* markSceneChanged: the next bte_render resets accumulation first */
/* The last frame as a PNG, top row first (the framebuffer's row 0 is the bottom row, as in the reference's
 * pixel buffer; captureScreenshot flips it the same way). */
int bte_write_png(const char* path);
/* captureScreenshot: screenshot_0000.png, _0001, ... in the working directory; the name goes to nameOut. */
int bte_capture_screenshot(char* nameOut, int nameCapacity);
/* startRecording / per-frame capture / stopRecording.  rawPath NULL: the reference's FFmpeg pipe (output.mp4,
 * H.264, `fps` playback); otherwise raw RGBA frames, rows bottom first, appended to that file per call of
 * bte_record_frame. */
int bte_record_start(const char* rawPath, int fps);
int bte_record_frame(void);
int bte_record_stop(void);
/* RGBA8 rows (first row first) -> PNG bytes; with out NULL only *size is set. */
int bte_encode_png(const uint8_t* rgba, int width, int height, uint8_t* out, long long capacity, long long* size);

/* ---- glTF 2.0 / GLB models: loadGltfModel (include/gltf_loader.h:25-30, src/gltf_loader.cpp:768-846) ----
 * Triangles (with the <model> transform posX/Y/Z, rotX/Y/Z degrees, scaleX/Y/Z applied after the node graph;
 * NULL = identity), per-triangle material slots, and per slot a Disney BSDF, emission and RGBA8 albedo /
 * metallic-roughness images (width = height = 0 when absent).  bte_scene_load reads <model> entries with it. */
typedef struct BteGltf BteGltf;
int bte_gltf_load(const char* path, const float* transform9, BteGltf** out);
int bte_gltf_counts(const BteGltf* model, int* triangles, int* materials, int* skippedOutliers);
int bte_gltf_triangles(const BteGltf* model, TriangleData* triangles, int* materialIds);
int bte_gltf_material(const BteGltf* model, int index, BsdfData* bsdf, float* emission3, int* isEmitter,
                      int* albedoWidthHeight, int* mrWidthHeight, uint8_t* albedoRGBA, uint8_t* mrRGBA);
void bte_gltf_free(BteGltf* model);

/* ---- scene.xml / OBJ loader (src/scene.cpp:83-523, src/main.cpp:267-930) ---- */
typedef struct BteScene BteScene;
typedef struct {
    const TriangleData* triangles; int triangleCount;
    const Float3* materials; int materialCount;
    const int* triangleMaterialIds;
    const int* triangleBsdfIds;
    const BsdfData* bsdfs; int bsdfCount;
    const Float3* triangleEmission;
    const uint8_t* triangleEmitterFlags;
    const EmitterData* emitters; int emitterCount;
    const int* emitterTriIndices; int emitterTriIndexCount;
    const float* emitterTriCdf; int emitterTriCdfCount;
    const float* sceneEmitterCdf;
    const SpotlightData* spotlights; int spotlightCount;
    const float* envRGBA; int envWidth, envHeight; float envIntensity, envRotationDeg;
    CameraData camera;
    int width, height;
    /* per material (count = materialCount): RGBA8 albedo / metallic-roughness images, NULL where a material
     * has none, with their sizes (1 x 1 for none): the arguments of bte_init_textures / bte_init_mr_textures */
    const uint8_t* const* albedoPixels; const int* albedoWidths; const int* albedoHeights;
    const uint8_t* const* mrPixels; const int* mrWidths; const int* mrHeights;
} BteSceneArrays;
/* PNG or JPEG bytes -> RGBA8, rows top to bottom, the decoding stbi_load(..., 4) gives the reference's
 * textures (src/main.cpp:407-470).  With outRGBA NULL only the size and the file's channel count are
 * returned; otherwise `capacity` must hold width*height*4 bytes. */
int bte_image_decode(const uint8_t* bytes, long long size, uint8_t* outRGBA, long long capacity, int* width,
                     int* height, int* channelsInFile);
int bte_scene_load(const char* scenePath, BteScene** out);
int bte_scene_arrays(const BteScene* scene, BteSceneArrays* out);
void bte_scene_free(BteScene* scene);
int bte_scene_upload(const BteScene* scene);   /* all bte_init_* calls of src/main.cpp:819-930 in order */

#ifdef __cplusplus
}
#endif
#endif
