// bte_renderer.cu -- renderer state and the C-ABI entry points.
//
// Host orchestration of the reference (src/render_kernel.cu,
// src/host/scene_upload.cu, src/host/wavefront_host.cu,
// src/host/renderer_state.*) restated for one B200: one process-wide renderer
// state (the reference's s_* globals), one stream, device-resident uploads,
// an LBVH instead of the OptiX GAS, and a frame that is a fixed,
// host-synchronisation-free launch sequence.  Every entry point returns a
// status and records a message for bte_last_error() instead of exiting.
#include "../../include/bte/launch_params.h"
#include "bte_denoise.h"
#include "bte_internal.h"
#include "bte_kernels.h"
#include "bte_math.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace bte {

namespace {

thread_local std::string g_lastError;

struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct CudaError {
    std::string msg;
};

inline void ck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw CudaError{std::string(what) + ": " + cudaGetErrorString(e)};
}

void upload(DeviceBuffer& b, const void* src, size_t bytes, cudaStream_t st)
{
    b.release();
    if (!src || bytes == 0) return;
    ck(cudaMalloc(&b.p, bytes), "cudaMalloc");
    b.bytes = bytes;
    ck(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync H2D");
}

void ensure(DeviceBuffer& b, size_t bytes)
{
    if (b.p && b.bytes >= bytes) return;
    b.release();
    if (bytes == 0) return;
    ck(cudaMalloc(&b.p, bytes), "cudaMalloc");
    b.bytes = bytes;
}

struct Renderer {
    bool init = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;         // shadow-ray stage of a bounce, beside the next bounce's extend
    cudaEvent_t evShade = nullptr, evConnect = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t stageEv[8] = {};

    // scene (src/host/renderer_state.h:30-169)
    DeviceBuffer tris, materials, triMatIds, emission, emitterFlags, triEmitter, emitters, emitterTriIndices,
        emitterTriCdf, sceneEmitterCdf, bsdfs, triBsdfIds, spots;
    int triCount = 0, materialCount = 0, emitterCount = 0, bsdfCount = 0, spotCount = 0;
    float sceneMaxAbs = 0.0f;
    bool hasEmission = false, hasFlags = false;
    std::vector<int> hostEmitterTriIndices;
    std::vector<EmitterData> hostEmitters;
    // textures
    std::vector<DeviceBuffer> tex, texMr;
    DeviceBuffer texTable, texTableMr;
    int textureCount = 0;
    bool hasMr = false;
    // env map
    DeviceBuffer envTexels, envMarginal, envConditional, envRowProb, envRowAlias, envColProb, envColAlias, envPixelPdf;
    int envW = 0, envH = 0;
    float envIntensity = 0.0f, envRotation = 0.0f, envTotalPowerF = 0.0f;
    double envTotalPowerD = 0.0;
    bool hasEnv = false;
    // acceleration structure
    DeviceBuffer bvhNodes, wideNodes, leafTris;
    int rootIsLeaf = 0, rootCode = ~0;
    int maxLeaf = 2;          // autotuned on B200 (8-wide tree, 1.04M-triangle scene): up to 2 triangles per leaf
    int bvhWidth = 8;         // tree built by the next bte_init_accel
    int postponePct = 0;      // 8-wide walk: leaf-test postponing threshold (0: never; neutral on the bench scene)
    int sortShading = 1;      // material-sorted shading (shade 5.9 -> 2.6 ms per frame on the 1080p bench scene)
    int tailPaths = 4096;     // bounce queues shorter than this finish in the tail kernel (eight lanes per path)
    int bvhBuilder = 1;       // binary hierarchy of the next bte_init_accel: 0 Morton-prefix (Karras), 1 PLOC
                              // (PLOC: frame 10.96 -> 10.54 ms on the 1080p bench scene)
    int wideCollapse = 1;     // 8-wide node children: 0 greedy by surface area, 1 surface-area-optimal (DP)
    int plocRadius = 4;       // PLOC neighbour search radius (measured on the 1080p scene: 4 best of 4/6/8/12/16/32)
    int builtBuilder = 0;     // hierarchy in use
    int overlapConnect = 1;   // bounce b's shadow rays run beside bounce b+1's closest-hit rays (11.1 -> 9.5 ms)
    int leafTestsPerStep = 0; // 8-wide walk: triangle tests per step (0: all of a node's leaves at once)
    int orderBounces = 3;     // leading bounces whose buckets and queues are rebuilt in path order (0: off)
    int raySortBits = 0;      // ray reordering before extend: origin cell bits per axis (0: off)
    int raySortBounces = 4;   // bounces 1..raySortBounces are reordered
    bool sceneChanged = false;   // bte_mark_scene_changed: the next bte_render resets accumulation first
    int builtWidth = 2;       // tree in use
    int accelNodes = 0, accelDepth = 0;
    int shadeMinBlocks = 3;   // autotuned on B200: 3 resident shade blocks per SM
    bool accelReady = false;
    float msBvh = 0.0f;
    // camera / frame
    CameraData camera{};
    BteRenderConfig cfg{1, 200, 3, BTE_ENV_SAMPLING_CDF, 128, 0};
    int renderMode = BTE_RENDER_WAVEFRONT;
    bool denoiser = false;
    uint32_t frameIndex = 0;
    int accumW = 0, accumH = 0;
    DeviceBuffer accum, accumD, framebuffer;
    uint32_t* extFramebuffer = nullptr;
    // wavefront buffers
    DeviceBuffer pO, pD, pTp, pL, pHit, q0, q1, rayCount, shadowCount, fetch, shadowQueue, shOrigin, shDir, shContrib,
        shMask, hitLog, errorFlags, sortQueue, sortCount, rayBin, sortedQueue, binCount, pathKey, orderStatus,
        orderTicket;
    int pathCap = 0, slotCap = 0, depthCap = 0;
    bool hitLogEnabled = false;
    bool aovEnabled = false;          // albedo / normal features for the denoiser
    DeviceBuffer aovAlbedo, aovNormal, aovAccum;
    DeviceBuffer denoised;            // [W*H*3] denoised mean radiance of the last frame (denoiser on)
    // batched views (bte_render_views): accumulation per view slot
    struct ViewState {
        int w = 0, h = 0;
        uint32_t frameIndex = 0;
        DeviceBuffer accum, accumD, fb;
    };
    std::vector<ViewState> views;
    DeviceBuffer viewTable;
    ViewDesc* hViewTable = nullptr;   // pinned staging of the view table: its upload does not block the host
    int pendDepth = 0, pendPaths = 0, pendCount = 0;   // a view frame enqueued and not yet finished
    // captured view frame (memsets, generate, bounces, tail, present) and its key; viewGen numbers captures
    cudaGraph_t viewGraph = nullptr;
    cudaGraphExec_t viewExec = nullptr;
    std::vector<unsigned char> viewKey;
    unsigned long long viewGen = 0;
    bool stageTiming = false;
    int lastPaths = 0, lastDepth = 0, lastSpp = 0, lastW = 0, lastH = 0, lastSlots = 0;
    BteFrameStats stats{};
    int gridExtend = 0, gridShade = 0, gridConnect = 0, gridBlock = 0;
    // frame index read by the kernels from device memory (pinned host word -> device word each frame)
    uint32_t* hFrameIndex = nullptr;
    DeviceBuffer dFrameIndex;
    // captured frame (memsets, generate, the bounce loop, present) and the launch parameters it was captured with
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    std::vector<unsigned char> graphKey;
};

// Scene slots: the selected slot's state lives in g, the others are parked in g_parked (the selected
// slot's own entry there is empty).  Every upload and render entry point acts on g.
constexpr int kMaxScenes = 8;
Renderer g;
Renderer g_parked[kMaxScenes];
int g_scene = 0;
std::mutex g_mutex;
constexpr int kMaxViews = 64;
constexpr int kMegakernelSpp = 5;   // SAMPLES_PER_PIXEL, include/rt_constants.cuh:11

void selectScene(int k)
{
    if (k < 0 || k >= kMaxScenes) throw CudaError{"bte_select_scene: scene slot out of range (0..7)"};
    if (k == g_scene) return;
    std::swap(g, g_parked[g_scene]);
    std::swap(g, g_parked[k]);
    g_scene = k;
}

// A batch of scenes whose view frames are all captured: one parent graph holding each scene's view graph as a
// child node (no edges between them), launched once on its own stream.
struct BatchGraph {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned long long> key;   // (slot, capture number) per child
};
BatchGraph g_batch;
unsigned long long g_captures = 0;

void ensureInit()
{
    if (g.init) return;
    int n = 0;
    ck(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (n <= 0) throw CudaError{"no CUDA device"};
    ck(cudaGetDevice(&g.device), "cudaGetDevice");
    ck(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaStreamCreateWithFlags(&g.side, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&g.evShade, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&g.evConnect, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreate(&g.ev0), "cudaEventCreate");
    ck(cudaEventCreate(&g.ev1), "cudaEventCreate");
    for (auto& e : g.stageEv) ck(cudaEventCreate(&e), "cudaEventCreate");
    ck(cudaHostAlloc(reinterpret_cast<void**>(&g.hFrameIndex), sizeof(uint32_t), cudaHostAllocDefault), "cudaHostAlloc");
    ensure(g.dFrameIndex, sizeof(uint32_t));
    std::string err;
    if (prepareEnvNoallocScratch(err) != 0) throw CudaError{err};
    g.init = true;
}

DevScene makeDevScene()
{
    DevScene s;
    std::memset(&s, 0, sizeof(s));   // padding too: the struct's bytes key the captured frame graph
    s.tris = g.tris.as<TriangleData>();
    s.triCount = g.accelReady ? g.triCount : 0;
    s.leafTris = g.leafTris.as<float4>();
    s.nodes = g.bvhNodes.as<BvhNode>();
    s.wnodes = g.wideNodes.as<WideNode>();
    s.bvhWidth = g.builtWidth;
    s.wideNodeCount = g.builtWidth == 8 ? g.accelNodes : 0;
    s.postponePct = g.postponePct;
    s.leafTestsPerStep = g.leafTestsPerStep;
    s.rootIsLeaf = g.rootIsLeaf;
    s.rootCode = g.rootCode;
    s.sceneMaxAbs = g.sceneMaxAbs;
    s.bsdfs = g.bsdfs.as<BsdfData>();
    s.triBsdfIds = g.triBsdfIds.as<int>();
    s.triMaterialIds = g.triMatIds.as<int>();
    s.texTable = g.textureCount > 0 ? g.texTable.as<TexRef>() : nullptr;
    s.texTableMr = (g.textureCount > 0 && g.hasMr) ? g.texTableMr.as<TexRef>() : nullptr;
    s.textureCount = g.textureCount;
    s.emitterFlags = g.emitterFlags.as<uint8_t>();
    s.emission = g.emission.as<Float3>();
    s.triEmitter = g.triEmitter.as<int>();
    s.emitters = g.emitters.as<EmitterData>();
    s.emitterCount = g.emitterCount;
    s.emitterTriIndices = g.emitterTriIndices.as<int>();
    s.emitterTriCdf = g.emitterTriCdf.as<float>();
    s.sceneEmitterCdf = g.sceneEmitterCdf.as<float>();
    s.spots = g.spots.as<SpotlightData>();
    s.spotCount = g.spotCount;
    s.hasEnv = g.hasEnv ? 1 : 0;
    DevEnv& e = s.env;
    e.texels = g.envTexels.as<float4>();
    e.w = g.envW; e.h = g.envH;
    e.intensity = g.envIntensity;
    e.rotation = g.envRotation;
    e.sampling = g.cfg.envSampling;
    e.totalPower = (g.cfg.envSampling == BTE_ENV_SAMPLING_ALIAS) ? static_cast<float>(g.envTotalPowerD) : g.envTotalPowerF;
    e.marginal = g.envMarginal.as<float>();
    e.conditional = g.envConditional.as<float>();
    e.rowProb = g.envRowProb.as<float>();
    e.rowAlias = g.envRowAlias.as<int>();
    e.colProb = g.envColProb.as<float>();
    e.colAlias = g.envColAlias.as<int>();
    e.pixelPdf = g.envPixelPdf.as<float>();
    return s;
}

// The tri -> emitter side table: for each triangle the first emitter (in
// emitter order) whose list holds it, as findEmitterIndexForTriangle
// (include/rt_emitter_sampling.cuh:132-148) returns.
void rebuildTriEmitter()
{
    g.triEmitter.release();
    if (g.triCount <= 0 || g.emitterCount <= 0) return;
    std::vector<int> t(static_cast<size_t>(g.triCount), -1);
    for (int e = g.emitterCount - 1; e >= 0; --e) {
        const EmitterData& E = g.hostEmitters[static_cast<size_t>(e)];
        for (int j = 0; j < E.triCount; ++j) {
            const size_t k = static_cast<size_t>(E.triIndexOffset) + static_cast<size_t>(j);
            if (k >= g.hostEmitterTriIndices.size()) continue;
            const int ti = g.hostEmitterTriIndices[k];
            if (ti >= 0 && ti < g.triCount) t[static_cast<size_t>(ti)] = e;
        }
    }
    upload(g.triEmitter, t.data(), t.size() * sizeof(int), g.stream);
}

void releaseGraph()
{
    if (g.graphExec) cudaGraphExecDestroy(g.graphExec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.graphExec = nullptr;
    g.graph = nullptr;
    g.graphKey.clear();
}

void releaseViewGraph()
{
    if (g.viewExec) cudaGraphExecDestroy(g.viewExec);
    if (g.viewGraph) cudaGraphDestroy(g.viewGraph);
    g.viewExec = nullptr;
    g.viewGraph = nullptr;
    g.viewKey.clear();
}

void releaseWavefront()
{
    releaseGraph();
    releaseViewGraph();
    for (DeviceBuffer* b : {&g.pO, &g.pD, &g.pTp, &g.pL, &g.pHit, &g.q0, &g.q1, &g.rayCount, &g.shadowCount, &g.fetch,
                            &g.sortQueue, &g.sortCount, &g.shadowQueue, &g.rayBin, &g.sortedQueue, &g.binCount,
                            &g.pathKey, &g.orderStatus, &g.orderTicket,
                            &g.shOrigin, &g.shDir, &g.shContrib, &g.shMask, &g.hitLog, &g.errorFlags})
        b->release();
    g.aovAlbedo.release(); g.aovNormal.release();
    g.pathCap = g.slotCap = g.depthCap = 0;
}

// bin counts of the reordered bounces (0..raySortBounces) for the current ray-sort setting
size_t rayBinBytes() { return sizeof(int) * static_cast<size_t>(g.raySortBounces + 1) * (8u << (3 * g.raySortBits)); }

// ray-reordering fields of a frame's DevPaths (off in megakernel mode)
void setRaySort(DevPaths& P, bool on)
{
    if (!on || g.raySortBits <= 0) return;
    P.rayBin = g.rayBin.as<int>();
    P.binCount = g.binCount.as<int>();
    P.sortedQueue = g.sortedQueue.as<int>();
    P.raySortBits = g.raySortBits;
    P.raySortBounces = g.raySortBounces;
}

// look-back words of a frame's ordered compactions (two per ordered bounce) over `paths` paths
size_t orderStatusBytes(int paths)
{
    return static_cast<size_t>(2 * g.orderBounces) * orderTiles(paths) * kSortKeys * sizeof(unsigned long long);
}

// path-ordered queue fields of a frame's DevPaths (off in megakernel mode, without material-sorted shading and
// with ray reordering, which appends the next queue in bin order)
void setOrder(DevPaths& P, bool on)
{
    if (!on || g.orderBounces <= 0 || !P.sortQueue || P.raySortBits > 0) return;
    P.pathKey = g.pathKey.as<uint8_t>();
    P.orderStatus = g.orderStatus.as<unsigned long long>();
    P.orderTicket = g.orderTicket.as<int>();
    P.orderBounces = g.orderBounces;
}

// frame prologue of the ordered compactions: clear their tickets and look-back words
void clearOrder(const DevPaths& P, cudaStream_t st)
{
    if (P.orderBounces <= 0) return;
    ck(cudaMemsetAsync(g.orderStatus.p, 0, orderStatusBytes(P.count), st), "cudaMemsetAsync");
    ck(cudaMemsetAsync(g.orderTicket.p, 0, sizeof(int) * 2 * P.orderBounces, st), "cudaMemsetAsync");
}

void ensureWavefront(int paths, int slots, int depth)
{
    const bool grow = paths > g.pathCap || slots > g.slotCap || depth > g.depthCap;
    const size_t binBytes = g.raySortBits > 0 ? rayBinBytes() : 0;
    if (!grow && (!g.hitLogEnabled || g.hitLog.p) && (!g.sortShading || g.sortQueue.p) &&
        (!g.raySortBits || (g.sortedQueue.p && g.binCount.bytes >= binBytes)) &&
        (!g.orderBounces || (g.pathKey.p && g.orderStatus.bytes >= orderStatusBytes(g.pathCap))))
        return;
    if (grow) {
        releaseWavefront();
        const size_t P = static_cast<size_t>(paths), S = static_cast<size_t>(slots);
        ensure(g.pO, P * 16); ensure(g.pD, P * 16); ensure(g.pTp, P * 16); ensure(g.pL, P * 16); ensure(g.pHit, P * 16);
        ensure(g.q0, P * 4); ensure(g.q1, P * 4);
        ensure(g.rayCount, sizeof(int) * (depth + 1));
        ensure(g.shadowCount, sizeof(int) * (depth + 1));
        ensure(g.fetch, sizeof(int) * 2 * (depth + 1));
        ensure(g.sortCount, sizeof(int) * kSortKeys * (depth + 1));
        ensure(g.shadowQueue, P * S * 4);
        ensure(g.shOrigin, P * 16);
        ensure(g.shDir, P * S * 16);
        ensure(g.shContrib, P * S * 16);
        ensure(g.shMask, P * 4);
        ensure(g.errorFlags, 4);
        g.pathCap = paths; g.slotCap = slots; g.depthCap = depth;
    }
    if (g.hitLogEnabled) ensure(g.hitLog, static_cast<size_t>(g.pathCap) * g.depthCap * 4);
    if (g.sortShading) ensure(g.sortQueue, static_cast<size_t>(g.pathCap) * kSortKeys * 4);
    if (g.orderBounces > 0) {
        if (!g.pathKey.p) {   // keys padded to whole tiles, padding never written
            const size_t bytes = static_cast<size_t>(orderTiles(g.pathCap)) * kOrderTile;
            ensure(g.pathKey, bytes);
            ck(cudaMemset(g.pathKey.p, kKeyDead, bytes), "cudaMemset");
        }
        ensure(g.orderStatus, orderStatusBytes(g.pathCap));
        ensure(g.orderTicket, sizeof(int) * 2 * 64);
    }
    if (g.raySortBits > 0) {
        ensure(g.rayBin, static_cast<size_t>(g.pathCap) * 4);
        ensure(g.sortedQueue, static_cast<size_t>(g.pathCap) * 4);
        ensure(g.binCount, binBytes);
    }
}

void ensureAov(int paths)
{
    if (!g.aovEnabled) return;
    if (g.aovAlbedo.bytes < static_cast<size_t>(paths) * 16) {
        g.aovAlbedo.release(); g.aovNormal.release();
        ensure(g.aovAlbedo, static_cast<size_t>(paths) * 16);
        ensure(g.aovNormal, static_cast<size_t>(paths) * 16);
    }
    const size_t n = static_cast<size_t>(g.accumW) * g.accumH * 6 * sizeof(float);
    if (g.aovAccum.bytes != n) {
        g.aovAccum.release();
        ensure(g.aovAccum, n);
        ck(cudaMemsetAsync(g.aovAccum.p, 0, n, g.stream), "cudaMemsetAsync");
    }
}

void ensureAccum(int w, int h)
{
    const size_t n = static_cast<size_t>(w) * h;
    if (g.accumW != w || g.accumH != h || !g.accum.p) {
        g.accum.release(); g.accumD.release(); g.framebuffer.release();
        ensure(g.accum, n * 12);
        ensure(g.accumD, n * 24);
        ensure(g.framebuffer, n * 4);
        g.accumW = w; g.accumH = h;
    }
    ck(cudaMemsetAsync(g.accum.p, 0, n * 12, g.stream), "cudaMemsetAsync");
    ck(cudaMemsetAsync(g.accumD.p, 0, n * 24, g.stream), "cudaMemsetAsync");
    ck(cudaMemsetAsync(g.framebuffer.p, 0, n * 4, g.stream), "cudaMemsetAsync");
    if (g.aovAccum.p) {
        if (g.aovAccum.bytes == n * 24) ck(cudaMemsetAsync(g.aovAccum.p, 0, n * 24, g.stream), "cudaMemsetAsync");
        else g.aovAccum.release();
    }
    ck(cudaStreamSynchronize(g.stream), "cudaStreamSynchronize");
    g.frameIndex = 0;
}

int slotsFor() { return 1 + g.spotCount + 1; }

// The bounce loop.  Bounce b's shadow rays (connect) only clear visibility bits that bounce b+1's shade
// reads, and bounce b+1's closest-hit rays (extend) only need bounce b's shade, so with overlapConnect
// connect(b) runs on the side stream beside extend(b+1): shade(b) -> {connect(b) | extend(b+1)} ->
// shade(b+1).  The few-ray launches of the last bounces are latency-bound, and the two overlap there.
void launchBounces(const DevScene& s, const DevPaths& P, const FrameParams& f, int depth, int block, cudaStream_t st)
{
    for (int b = 0; b < depth; ++b) {
        if (P.raySortBits > 0 && b >= 1 && b <= P.raySortBounces) launchRaySort(P, b, g.gridShade, st);
        launchExtend(s, P, b, g.gridExtend, block, st);
        if (b < P.orderBounces) launchOrder(P, b, false, st);
        if (g.overlapConnect && b > 0) ck(cudaStreamWaitEvent(st, g.evConnect, 0), "cudaStreamWaitEvent");
        launchShade(s, P, f, b, g.gridShade, block, g.shadeMinBlocks, st);
        const bool orderNext = b + 1 < P.orderBounces && b + 1 < depth;
        if (g.overlapConnect) {
            ck(cudaEventRecord(g.evShade, st), "cudaEventRecord");
            ck(cudaStreamWaitEvent(g.side, g.evShade, 0), "cudaStreamWaitEvent");
            launchConnect(s, P, b, g.gridConnect, block, g.side);
            ck(cudaEventRecord(g.evConnect, g.side), "cudaEventRecord");
            if (orderNext) launchOrder(P, b, true, st);
        } else {
            if (orderNext) launchOrder(P, b, true, st);
            launchConnect(s, P, b, g.gridConnect, block, st);
        }
    }
    if (g.overlapConnect && depth > 0) ck(cudaStreamWaitEvent(st, g.evConnect, 0), "cudaStreamWaitEvent");
}

void renderFrame(int w, int h)
{
    if (w <= 0 || h <= 0) throw CudaError{"bte_render: image size must be positive"};
    if (!g.tris.p || g.triCount <= 0) throw CudaError{"bte_render: no scene uploaded (bte_init_scene)"};
    if (!g.accelReady) throw CudaError{"bte_render: acceleration structure missing (call bte_init_accel after bte_init_scene)"};
    if (!g.bsdfs.p || !g.triBsdfIds.p) throw CudaError{"bte_render: no BSDFs uploaded (bte_init_bsdfs)"};
    if (!g.emitterFlags.p) throw CudaError{"bte_render: emitter flags missing (bte_init_triangle_emitter_flags)"};
    if (!g.accum.p || g.accumW != w || g.accumH != h) ensureAccum(w, h);   // render_kernel.cu:62-64
    // megakernel mode: SAMPLES_PER_PIXEL (rt_constants.cuh:11) paths per pixel on one stream, one path slot a pixel
    const bool mega = g.renderMode == BTE_RENDER_MEGAKERNEL;
    const int spp = mega ? kMegakernelSpp : (g.cfg.samplesPerFrame > 0 ? g.cfg.samplesPerFrame : 1);
    const int depth = g.cfg.maxDepth > 0 ? g.cfg.maxDepth : 1;
    const long long paths64 = static_cast<long long>(w) * h * (mega ? 1 : spp);
    if (paths64 > (1LL << 30)) throw CudaError{"bte_render: too many paths per frame (W*H*spp > 2^30)"};
    const int paths = static_cast<int>(paths64);
    const int slots = slotsFor();
    if (slots > 32) throw CudaError{"bte_render: at most 30 spotlights are supported"};
    ensureWavefront(paths, slots, depth);
    ensureAov(paths);
    const int block = g.cfg.blockSize > 0 ? g.cfg.blockSize : 128;
    if (g.gridBlock != block) {
        g.gridExtend = occupancyGrid(g.builtWidth == 8 ? 4 : 0, block);
        g.gridShade = occupancyGrid(g.shadeMinBlocks == 4 ? 6 : g.shadeMinBlocks == 3 ? 3 : 1, block);
        g.gridConnect = occupancyGrid(g.builtWidth == 8 ? 5 : 2, block);
        g.gridBlock = block;
    }
    DevPaths P;
    std::memset(&P, 0, sizeof(P));
    P.o = g.pO.as<float4>(); P.d = g.pD.as<float4>(); P.tp = g.pTp.as<float4>(); P.L = g.pL.as<float4>();
    P.hit = g.pHit.as<float4>();
    P.queue[0] = g.q0.as<int>(); P.queue[1] = g.q1.as<int>();
    P.rayCount = g.rayCount.as<int>();
    P.shadowCount = g.shadowCount.as<int>();
    P.fetch = g.fetch.as<int>();
    P.shadowQueue = g.shadowQueue.as<int>();
    P.shOrigin = g.shOrigin.as<float4>();
    P.shDir = g.shDir.as<float4>();
    P.shContrib = g.shContrib.as<float4>();
    P.shMask = g.shMask.as<uint32_t>();
    P.hitLog = g.hitLogEnabled && !mega ? g.hitLog.as<int>() : nullptr;
    P.aovAlbedo = g.aovEnabled ? g.aovAlbedo.as<float4>() : nullptr;
    P.aovNormal = g.aovEnabled ? g.aovNormal.as<float4>() : nullptr;
    P.slots = slots;
    P.maxDepth = depth;
    P.count = paths;
    P.errorFlags = g.errorFlags.as<unsigned int>();
    P.sortQueue = g.sortShading ? g.sortQueue.as<int>() : nullptr;
    P.sortCount = g.sortCount.as<int>();
    P.tailPaths = mega ? 0 : g.tailPaths;
    setRaySort(P, !mega);
    setOrder(P, !mega);
    FrameParams f;
    std::memset(&f, 0, sizeof(f));
    f.width = w; f.height = h; f.spp = spp;
    f.frameIndex = g.dFrameIndex.as<uint32_t>();
    f.rrStart = g.cfg.rrStart;
    f.tanHalf = m::tanf_(0.5f * g.camera.fovYRadians);
    f.cam = g.camera;
    const DevScene s = makeDevScene();
    cudaStream_t st = g.stream;
    *g.hFrameIndex = g.frameIndex;   // the previous frame synchronised, so no copy still reads this word
    float* accumF = g.accum.as<float>();
    double* accumDv = g.accumD.as<double>();
    uint32_t* fb = g.framebuffer.as<uint32_t>();
    float* aovAcc = g.aovEnabled ? g.aovAccum.as<float>() : nullptr;
    auto prologue = [&] {
        ck(cudaMemsetAsync(g.rayCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.shadowCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.fetch.p, 0, sizeof(int) * 2 * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.sortCount.p, 0, sizeof(int) * kSortKeys * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.errorFlags.p, 0, 4, st), "cudaMemsetAsync");
        if (P.raySortBits > 0) ck(cudaMemsetAsync(g.binCount.p, 0, rayBinBytes(), st), "cudaMemsetAsync");
        clearOrder(P, st);
        if (g.hitLogEnabled) ck(cudaMemsetAsync(g.hitLog.p, 0xfe, static_cast<size_t>(paths) * depth * 4, st), "cudaMemsetAsync");
        ck(cudaMemcpyAsync(g.dFrameIndex.p, g.hFrameIndex, sizeof(uint32_t), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
    };
    auto frameLaunches = [&] {
        if (mega) {
            launchMegakernel(s, P, f, accumF, accumDv, fb, g.extFramebuffer, aovAcc, st);
            return;
        }
        launchGenerate(P, f, st);
        launchBounces(s, P, f, depth, block, st);
        launchTail(s, P, f, st);
        launchPresent(P, f, accumF, accumDv, fb, g.extFramebuffer, aovAcc, st);
    };
    float stage[6] = {0, 0, 0, 0, 0, 0};
    if (g.cfg.useGraph && (!g.stageTiming || mega)) {
        // One graph per launch configuration: every kernel argument is part of the key, so a change of
        // scene, buffers, image size, depth or tuning re-captures; the frame index travels through memory.
        std::vector<unsigned char> key;
        auto put = [&](const void* p, size_t n) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            key.insert(key.end(), c, c + n);
        };
        const int ints[9] = {depth, block, g.gridExtend, g.gridShade, g.gridConnect, g.shadeMinBlocks, paths,
                             g.hitLogEnabled ? 1 : 0, g.overlapConnect};
        const void* ptrs[5] = {accumF, accumDv, fb, g.extFramebuffer, aovAcc};
        put(&P, sizeof(P)); put(&f, sizeof(f)); put(&s, sizeof(s)); put(ints, sizeof(ints)); put(ptrs, sizeof(ptrs));
        if (!g.graphExec || key != g.graphKey) {
            releaseGraph();
            ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            try {
                prologue();
                frameLaunches();
                ck(cudaGetLastError(), "kernel launch (capture)");
            } catch (...) {
                cudaGraph_t broken = nullptr;
                cudaStreamEndCapture(st, &broken);
                if (broken) cudaGraphDestroy(broken);
                throw;
            }
            ck(cudaStreamEndCapture(st, &g.graph), "cudaStreamEndCapture");
            ck(cudaGraphInstantiate(&g.graphExec, g.graph, 0), "cudaGraphInstantiate");
            g.graphKey = key;
        }
        ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
        ck(cudaGraphLaunch(g.graphExec, st), "cudaGraphLaunch");
    } else if (!g.stageTiming || mega) {
        ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
        prologue();
        frameLaunches();
    } else {
        prologue();
        ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
        // per-stage device time, summed over bounces (adds a sync per stage)
        auto timed = [&](int k, auto&& fn) {
            ck(cudaEventRecord(g.stageEv[0], st), "cudaEventRecord");
            fn();
            ck(cudaEventRecord(g.stageEv[1], st), "cudaEventRecord");
            ck(cudaEventSynchronize(g.stageEv[1]), "cudaEventSynchronize");
            float ms = 0.0f;
            ck(cudaEventElapsedTime(&ms, g.stageEv[0], g.stageEv[1]), "cudaEventElapsedTime");
            stage[k] += ms;
        };
        timed(0, [&] { launchGenerate(P, f, st); });
        for (int b = 0; b < depth; ++b) {
            timed(1, [&] {
                if (P.raySortBits > 0 && b >= 1 && b <= P.raySortBounces) launchRaySort(P, b, g.gridShade, st);
                launchExtend(s, P, b, g.gridExtend, block, st);
                if (b < P.orderBounces) launchOrder(P, b, false, st);
            });
            timed(2, [&] {
                launchShade(s, P, f, b, g.gridShade, block, g.shadeMinBlocks, st);
                if (b + 1 < P.orderBounces && b + 1 < depth) launchOrder(P, b, true, st);
            });
            timed(3, [&] { launchConnect(s, P, b, g.gridConnect, block, st); });
        }
        timed(5, [&] { launchTail(s, P, f, st); });
        timed(4, [&] { launchPresent(P, f, accumF, accumDv, fb, g.extFramebuffer, aovAcc, st); });
    }
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaEventRecord(g.ev1, st), "cudaEventRecord");
    std::vector<int> rc(static_cast<size_t>(depth + 1)), sc(static_cast<size_t>(depth + 1));
    unsigned int errFlags = 0;
    ck(cudaMemcpyAsync(rc.data(), g.rayCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(sc.data(), g.shadowCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(&errFlags, g.errorFlags.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(st), "frame");
    BteFrameStats& S = g.stats;
    S = BteFrameStats{};
    S.samples = mega ? paths64 * spp : paths;
    for (int b = 0; b < depth; ++b) {
        S.extends += rc[static_cast<size_t>(b)];
        S.shadowRays += sc[static_cast<size_t>(b)];
        if (rc[static_cast<size_t>(b)] > 0) S.maxBounceReached = b;
    }
    ck(cudaEventElapsedTime(&S.msTotal, g.ev0, g.ev1), "cudaEventElapsedTime");
    S.msGenerate = stage[0]; S.msExtend = stage[1]; S.msShade = stage[2]; S.msConnect = stage[3]; S.msPresent = stage[4];
    S.msTail = stage[5];
    S.tailBounce = -1;
    if (P.tailPaths > 0) {
        for (int b = 0; b < depth; ++b)
            if (rc[static_cast<size_t>(b)] < P.tailPaths) { S.tailBounce = b; break; }
        if (S.tailBounce >= 0)
            for (int b = S.tailBounce; b < depth; ++b) {
                S.tailExtends += rc[static_cast<size_t>(b)];
                S.tailShadowRays += sc[static_cast<size_t>(b)];
            }
    }
    if (g.denoiser && !(errFlags & 7u)) {
        const size_t bytes = static_cast<size_t>(w) * h * 12;
        if (g.denoised.bytes != bytes) { g.denoised.release(); ensure(g.denoised, bytes); }
        dn::denoiseForRenderer(accumF, aovAcc, 1, h, w, g.denoised.as<float>(), st);
        launchPackImage(g.denoised.as<float>(), w * h, fb, g.extFramebuffer, st);
        ck(cudaGetLastError(), "pack launch");
        ck(cudaStreamSynchronize(st), "denoise present");
    }
    g.frameIndex += mega ? 1u : static_cast<uint32_t>(spp);   // the megakernel counts frames
    g.lastPaths = mega ? 0 : paths; g.lastDepth = depth; g.lastSpp = spp; g.lastW = w; g.lastH = h; g.lastSlots = slots;
    if (errFlags & 1u) throw CudaError{"traversal stack overflow (BVH deeper than the traversal stack)"};
    if (errFlags & 2u) throw CudaError{"traversal met an out-of-range node or triangle index (malformed tree)"};
    if (errFlags & 4u) throw CudaError{"ordered queue compaction: a tile's wait for its predecessors gave up"};
}

// Several camera views of the scene in one frame: one launch sequence over the concatenated paths of all
// views (each view's paths sample-major as in bte_render), each view accumulating into its own buffers.
// launchViews only enqueues (no host wait once the buffers exist); finishViews waits for the frame and
// reads its counters, so several scenes' frames can be enqueued on their own streams before any wait.
void launchViews(const BteView* views, int count, bool deferToBatch = false)
{
    if (!views || count <= 0) throw CudaError{"bte_render_views: no views"};
    if (count > kMaxViews) throw CudaError{"bte_render_views: at most 64 views per frame"};
    if (!g.tris.p || g.triCount <= 0 || !g.accelReady || !g.bsdfs.p || !g.triBsdfIds.p || !g.emitterFlags.p)
        throw CudaError{"bte_render_views: scene, acceleration structure, BSDFs and emitter flags must be uploaded"};
    const int depth = g.cfg.maxDepth > 0 ? g.cfg.maxDepth : 1;
    const int slots = slotsFor();
    if (slots > 32) throw CudaError{"bte_render_views: at most 30 spotlights are supported"};
    if (static_cast<int>(g.views.size()) != count) g.views.resize(static_cast<size_t>(count));
    std::vector<ViewDesc> vd(static_cast<size_t>(count));
    long long paths64 = 0, pixels64 = 0;
    for (int v = 0; v < count; ++v) {
        const BteView& in = views[v];
        if (in.width <= 0 || in.height <= 0 || in.samplesPerFrame < 0)
            throw CudaError{"bte_render_views: view sizes must be positive and samplesPerFrame non-negative"};
        Renderer::ViewState& st = g.views[static_cast<size_t>(v)];
        const size_t n = static_cast<size_t>(in.width) * in.height;
        if (st.w != in.width || st.h != in.height || !st.accum.p) {   // new or resized view: fresh accumulation
            st.accum.release(); st.accumD.release(); st.fb.release();
            ensure(st.accum, n * 12); ensure(st.accumD, n * 24); ensure(st.fb, n * 4);
            ck(cudaMemsetAsync(st.accum.p, 0, n * 12, g.stream), "cudaMemsetAsync");
            ck(cudaMemsetAsync(st.accumD.p, 0, n * 24, g.stream), "cudaMemsetAsync");
            ck(cudaMemsetAsync(st.fb.p, 0, n * 4, g.stream), "cudaMemsetAsync");
            st.w = in.width; st.h = in.height; st.frameIndex = 0;
        }
        ViewDesc& d = vd[static_cast<size_t>(v)];
        std::memset(&d, 0, sizeof(d));
        d.cam = in.camera;
        d.tanHalf = m::tanf_(0.5f * in.camera.fovYRadians);
        d.width = in.width; d.height = in.height; d.spp = in.samplesPerFrame;
        d.frameIndex = st.frameIndex;
        d.pathOffset = static_cast<int>(paths64);
        d.pixelOffset = static_cast<int>(pixels64);
        d.accum = st.accum.as<float>(); d.accumD = st.accumD.as<double>(); d.framebuffer = st.fb.as<uint32_t>();
        paths64 += static_cast<long long>(n) * in.samplesPerFrame;
        pixels64 += static_cast<long long>(n);
        if (paths64 > (1LL << 30)) throw CudaError{"bte_render_views: too many paths per frame (sum W*H*spp > 2^30)"};
    }
    if (paths64 == 0) throw CudaError{"bte_render_views: every view has samplesPerFrame 0"};
    const int paths = static_cast<int>(paths64);
    ensureWavefront(paths, slots, depth);
    const int block = g.cfg.blockSize > 0 ? g.cfg.blockSize : 128;
    if (g.gridBlock != block) {
        g.gridExtend = occupancyGrid(g.builtWidth == 8 ? 4 : 0, block);
        g.gridShade = occupancyGrid(g.shadeMinBlocks == 4 ? 6 : g.shadeMinBlocks == 3 ? 3 : 1, block);
        g.gridConnect = occupancyGrid(g.builtWidth == 8 ? 5 : 2, block);
        g.gridBlock = block;
    }
    ensure(g.viewTable, sizeof(ViewDesc) * kMaxViews);
    if (!g.hViewTable)
        ck(cudaHostAlloc(reinterpret_cast<void**>(&g.hViewTable), sizeof(ViewDesc) * kMaxViews, cudaHostAllocDefault),
           "cudaHostAlloc");
    std::memcpy(g.hViewTable, vd.data(), sizeof(ViewDesc) * count);   // the previous view frame has finished
    ck(cudaMemcpyAsync(g.viewTable.p, g.hViewTable, sizeof(ViewDesc) * count, cudaMemcpyHostToDevice, g.stream),
       "cudaMemcpyAsync");
    DevPaths P;
    std::memset(&P, 0, sizeof(P));
    P.o = g.pO.as<float4>(); P.d = g.pD.as<float4>(); P.tp = g.pTp.as<float4>(); P.L = g.pL.as<float4>();
    P.hit = g.pHit.as<float4>();
    P.queue[0] = g.q0.as<int>(); P.queue[1] = g.q1.as<int>();
    P.rayCount = g.rayCount.as<int>();
    P.shadowCount = g.shadowCount.as<int>();
    P.fetch = g.fetch.as<int>();
    P.shadowQueue = g.shadowQueue.as<int>();
    P.shOrigin = g.shOrigin.as<float4>();
    P.shDir = g.shDir.as<float4>();
    P.shContrib = g.shContrib.as<float4>();
    P.shMask = g.shMask.as<uint32_t>();
    P.slots = slots;
    P.maxDepth = depth;
    P.count = paths;
    P.errorFlags = g.errorFlags.as<unsigned int>();
    P.sortQueue = g.sortShading ? g.sortQueue.as<int>() : nullptr;
    P.sortCount = g.sortCount.as<int>();
    // Batched views have no megakernel counterpart in the reference; in that mode every path of the views runs
    // start to end in the tail kernel (the wavefront's per-sample streams, bit-identical images).
    P.tailPaths = g.renderMode == BTE_RENDER_MEGAKERNEL ? 0x7fffffff : g.tailPaths;
    setRaySort(P, g.renderMode != BTE_RENDER_MEGAKERNEL);
    setOrder(P, g.renderMode != BTE_RENDER_MEGAKERNEL);
    FrameParams f;
    std::memset(&f, 0, sizeof(f));
    f.frameIndex = g.dFrameIndex.as<uint32_t>();
    f.rrStart = g.cfg.rrStart;
    f.views = g.viewTable.as<ViewDesc>();
    f.viewCount = count;
    const DevScene s = makeDevScene();
    cudaStream_t st = g.stream;
    auto body = [&] {
        ck(cudaMemsetAsync(g.rayCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.shadowCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.fetch.p, 0, sizeof(int) * 2 * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.sortCount.p, 0, sizeof(int) * kSortKeys * (depth + 1), st), "cudaMemsetAsync");
        ck(cudaMemsetAsync(g.errorFlags.p, 0, 4, st), "cudaMemsetAsync");
        if (P.raySortBits > 0) ck(cudaMemsetAsync(g.binCount.p, 0, rayBinBytes(), st), "cudaMemsetAsync");
        clearOrder(P, st);
        launchGenerate(P, f, st);
        launchBounces(s, P, f, depth, block, st);
        launchTail(s, P, f, st);
        launchPresentViews(P, f, static_cast<int>(pixels64), st);
    };
    const bool useGraph = g.cfg.useGraph != 0;
    if (useGraph) {
        // Every baked launch argument keys the capture; the view table's contents (cameras, per-view frame
        // indices, accumulation pointers) travel through device memory, uploaded before each launch.
        std::vector<unsigned char> key;
        auto put = [&](const void* p, size_t n) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            key.insert(key.end(), c, c + n);
        };
        const int ints[8] = {depth, block, g.gridExtend, g.gridShade, g.gridConnect, g.shadeMinBlocks,
                             static_cast<int>(pixels64), g.overlapConnect};
        put(&P, sizeof(P)); put(&f, sizeof(f)); put(&s, sizeof(s)); put(ints, sizeof(ints));
        if (!g.viewExec || key != g.viewKey) {
            releaseViewGraph();
            ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            try {
                body();
                ck(cudaGetLastError(), "kernel launch (capture)");
            } catch (...) {
                cudaGraph_t broken = nullptr;
                cudaStreamEndCapture(st, &broken);
                if (broken) cudaGraphDestroy(broken);
                throw;
            }
            ck(cudaStreamEndCapture(st, &g.viewGraph), "cudaStreamEndCapture");
            ck(cudaGraphInstantiate(&g.viewExec, g.viewGraph, 0), "cudaGraphInstantiate");
            g.viewKey = key;
            g.viewGen = ++g_captures;
        }
    }
    g.pendDepth = depth; g.pendPaths = paths; g.pendCount = count;
    if (deferToBatch) {   // the batch graph runs the captured frame; mark the table upload's end
        ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
        return;
    }
    ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
    if (useGraph)
        ck(cudaGraphLaunch(g.viewExec, st), "cudaGraphLaunch");
    else
        body();
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaEventRecord(g.ev1, st), "cudaEventRecord");
}

void finishViews(const BteView* views)
{
    const int depth = g.pendDepth, paths = g.pendPaths, count = g.pendCount;
    g.pendCount = 0;
    if (count <= 0) return;
    cudaStream_t st = g.stream;
    std::vector<int> rc(static_cast<size_t>(depth + 1)), sc(static_cast<size_t>(depth + 1));
    unsigned int errFlags = 0;
    ck(cudaMemcpyAsync(rc.data(), g.rayCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(sc.data(), g.shadowCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(&errFlags, g.errorFlags.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(st), "frame");
    BteFrameStats& S = g.stats;
    S = BteFrameStats{};
    S.samples = paths;
    S.tailBounce = -1;
    for (int b = 0; b < depth; ++b) {
        S.extends += rc[static_cast<size_t>(b)];
        S.shadowRays += sc[static_cast<size_t>(b)];
        if (rc[static_cast<size_t>(b)] > 0) S.maxBounceReached = b;
    }
    ck(cudaEventElapsedTime(&S.msTotal, g.ev0, g.ev1), "cudaEventElapsedTime");
    for (int v = 0; v < count; ++v)
        g.views[static_cast<size_t>(v)].frameIndex += static_cast<uint32_t>(views[v].samplesPerFrame);
    g.lastPaths = 0;   // per-path debug readbacks refer to single-view frames
    if (errFlags & 1u) throw CudaError{"traversal stack overflow (BVH deeper than the traversal stack)"};
    if (errFlags & 2u) throw CudaError{"traversal met an out-of-range node or triangle index (malformed tree)"};
    if (errFlags & 4u) throw CudaError{"ordered queue compaction: a tile's wait for its predecessors gave up"};
}

void renderViews(const BteView* views, int count)
{
    launchViews(views, count);
    finishViews(views);
}

// The batch as one graph launch: each scene's captured view frame is a child node of one parent graph (rebuilt
// when a scene re-captures), launched on the batch stream once every scene's view table is uploaded; each scene
// then reads its counters after the batch.  Every scene's frame time is the batch's.
void renderSceneBatchGraph(const int* scenes, const int* viewCounts, const BteView* views, int sceneCount,
                           const std::vector<int>& offset, int home)
{
    if (!g_batch.stream) {
        ck(cudaStreamCreateWithFlags(&g_batch.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaEventCreateWithFlags(&g_batch.done, cudaEventDisableTiming), "cudaEventCreate");
    }
    std::vector<unsigned long long> key;
    std::vector<cudaGraph_t> children;
    int prepared = 0;
    try {
        for (; prepared < sceneCount; ++prepared) {
            selectScene(scenes[prepared]);
            ensureInit();
            launchViews(views + offset[static_cast<size_t>(prepared)], viewCounts[prepared], true);
            ck(cudaStreamWaitEvent(g_batch.stream, g.ev0, 0), "cudaStreamWaitEvent");
            key.push_back(static_cast<unsigned long long>(scenes[prepared]));
            key.push_back(g.viewGen);
            children.push_back(g.viewGraph);
        }
        if (!g_batch.exec || key != g_batch.key) {
            if (g_batch.exec) cudaGraphExecDestroy(g_batch.exec);
            if (g_batch.graph) cudaGraphDestroy(g_batch.graph);
            g_batch.exec = nullptr;
            g_batch.graph = nullptr;
            g_batch.key.clear();
            ck(cudaGraphCreate(&g_batch.graph, 0), "cudaGraphCreate");
            for (cudaGraph_t child : children) {
                cudaGraphNode_t node;
                ck(cudaGraphAddChildGraphNode(&node, g_batch.graph, nullptr, 0, child), "cudaGraphAddChildGraphNode");
            }
            ck(cudaGraphInstantiate(&g_batch.exec, g_batch.graph, 0), "cudaGraphInstantiate");
            g_batch.key = key;
        }
        ck(cudaGraphLaunch(g_batch.exec, g_batch.stream), "cudaGraphLaunch");
        ck(cudaEventRecord(g_batch.done, g_batch.stream), "cudaEventRecord");
    } catch (const CudaError&) {
        for (int i = 0; i < prepared; ++i) {   // nothing of the batch ran: drop the pending frames
            selectScene(scenes[i]);
            g.pendCount = 0;
            cudaStreamSynchronize(g.stream);
        }
        selectScene(home);
        throw;
    }
    std::string firstError;
    for (int i = 0; i < sceneCount; ++i) {
        selectScene(scenes[i]);
        try {
            ck(cudaStreamWaitEvent(g.stream, g_batch.done, 0), "cudaStreamWaitEvent");
            ck(cudaEventRecord(g.ev1, g.stream), "cudaEventRecord");
            finishViews(views + offset[static_cast<size_t>(i)]);
        } catch (const CudaError& e) {
            if (firstError.empty()) firstError = e.msg;
        }
    }
    selectScene(home);
    if (!firstError.empty()) throw CudaError{firstError};
}

// Several scenes' views as one launch sequence (the default batch mode): the scene table and the per-path scene
// index, with the pinned staging of the scene and view tables and the captured frame.
struct FusedBatch {
    DeviceBuffer sceneTable, viewTable, pathScene;
    DevScene* hScenes = nullptr;   // [kMaxScenes]
    ViewDesc* hViews = nullptr;    // [kMaxScenes * kMaxViews]
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
};
FusedBatch g_fused;
int g_batchMode = 1;   // 1: one launch sequence over every scene's paths when the scenes allow it; 0: per scene

void releaseFusedGraph()
{
    if (g_fused.exec) cudaGraphExecDestroy(g_fused.exec);
    if (g_fused.graph) cudaGraphDestroy(g_fused.graph);
    g_fused.exec = nullptr;
    g_fused.graph = nullptr;
    g_fused.key.clear();
}

// One frame of several scenes' views in ONE launch sequence: the paths of every view of every scene are
// concatenated (scene by scene, view by view), each path carries its scene's index (written by generate), and
// the stage kernels take the path's geometry, tree, materials, lights and env map from the frame's scene table.
// The first scene's slot provides the path-state buffers, the stream and the frame-level settings (max depth,
// roulette start, block size, graph use, shading residency, material sorting, ray reordering, the shadow-ray
// overlap and the tail threshold).  The scenes must all render in wavefront mode with the 8-wide tree and share
// the first scene's max depth, roulette start, block size and graph use; otherwise nothing is done and false
// comes back (the caller then runs each scene's own launch sequence).  Every scene's views accumulate exactly as
// bte_render_views on that slot alone would leave them.
bool renderSceneBatchFused(const int* scenes, const int* viewCounts, const BteView* views, int sceneCount,
                           const std::vector<int>& offset, int home)
{
    if (g_batchMode == 0 || sceneCount < 2) return false;
    int depth = 1, rr = 3, block = 128, useGraph = 0, slots = 1;
    for (int i = 0; i < sceneCount; ++i) {   // eligibility first: nothing is changed unless the batch qualifies
        selectScene(scenes[i]);
        const int d = g.cfg.maxDepth > 0 ? g.cfg.maxDepth : 1;
        const int b = g.cfg.blockSize > 0 ? g.cfg.blockSize : 128;
        const bool ok = g.accelReady && g.builtWidth == 8 && g.renderMode == BTE_RENDER_WAVEFRONT &&
                        (i == 0 || (d == depth && g.cfg.rrStart == rr && b == block && g.cfg.useGraph == useGraph));
        if (!ok) {
            selectScene(home);
            return false;
        }
        if (i == 0) { depth = d; rr = g.cfg.rrStart; block = b; useGraph = g.cfg.useGraph; }
    }
    std::vector<ViewDesc> vd;
    std::vector<long long> sceneSamples(static_cast<size_t>(sceneCount), 0);
    DevScene table[kMaxScenes];
    std::memset(table, 0, sizeof(table));
    long long paths64 = 0, pixels64 = 0;
    try {
        for (int i = 0; i < sceneCount; ++i) {
            selectScene(scenes[i]);
            ensureInit();
            if (!g.tris.p || g.triCount <= 0 || !g.bsdfs.p || !g.triBsdfIds.p || !g.emitterFlags.p)
                throw CudaError{"bte_render_scene_batch: scene, acceleration structure, BSDFs and emitter flags must be uploaded"};
            slots = std::max(slots, slotsFor());
            if (slots > 32) throw CudaError{"bte_render_scene_batch: at most 30 spotlights are supported"};
            table[i] = makeDevScene();
            const BteView* sv = views + offset[static_cast<size_t>(i)];
            const int count = viewCounts[i];
            if (static_cast<int>(g.views.size()) != count) g.views.resize(static_cast<size_t>(count));
            for (int v = 0; v < count; ++v) {
                const BteView& in = sv[v];
                if (in.width <= 0 || in.height <= 0 || in.samplesPerFrame < 0)
                    throw CudaError{"bte_render_scene_batch: view sizes must be positive and samplesPerFrame non-negative"};
                Renderer::ViewState& st = g.views[static_cast<size_t>(v)];
                const size_t n = static_cast<size_t>(in.width) * in.height;
                if (st.w != in.width || st.h != in.height || !st.accum.p) {   // new or resized view: fresh accumulation
                    st.accum.release(); st.accumD.release(); st.fb.release();
                    ensure(st.accum, n * 12); ensure(st.accumD, n * 24); ensure(st.fb, n * 4);
                    ck(cudaMemsetAsync(st.accum.p, 0, n * 12, g.stream), "cudaMemsetAsync");
                    ck(cudaMemsetAsync(st.accumD.p, 0, n * 24, g.stream), "cudaMemsetAsync");
                    ck(cudaMemsetAsync(st.fb.p, 0, n * 4, g.stream), "cudaMemsetAsync");
                    st.w = in.width; st.h = in.height; st.frameIndex = 0;
                }
                ViewDesc d;
                std::memset(&d, 0, sizeof(d));
                d.cam = in.camera;
                d.tanHalf = m::tanf_(0.5f * in.camera.fovYRadians);
                d.width = in.width; d.height = in.height; d.spp = in.samplesPerFrame;
                d.frameIndex = st.frameIndex;
                d.pathOffset = static_cast<int>(paths64);
                d.pixelOffset = static_cast<int>(pixels64);
                d.scene = i;
                d.accum = st.accum.as<float>(); d.accumD = st.accumD.as<double>(); d.framebuffer = st.fb.as<uint32_t>();
                vd.push_back(d);
                paths64 += static_cast<long long>(n) * in.samplesPerFrame;
                pixels64 += static_cast<long long>(n);
                sceneSamples[static_cast<size_t>(i)] += static_cast<long long>(n) * in.samplesPerFrame;
                if (paths64 > (1LL << 30))
                    throw CudaError{"bte_render_scene_batch: too many paths per frame (sum W*H*spp > 2^30)"};
            }
            ck(cudaStreamSynchronize(g.stream), "cudaStreamSynchronize");   // new view buffers are cleared
        }
        if (paths64 == 0) throw CudaError{"bte_render_scene_batch: every view has samplesPerFrame 0"};
    } catch (...) {
        selectScene(home);
        throw;
    }
    selectScene(scenes[0]);
    const int paths = static_cast<int>(paths64), total = static_cast<int>(vd.size());
    try {
        ensureWavefront(paths, slots, depth);
        if (g.gridBlock != block) {
            g.gridExtend = occupancyGrid(4, block);
            g.gridShade = occupancyGrid(g.shadeMinBlocks == 4 ? 6 : g.shadeMinBlocks == 3 ? 3 : 1, block);
            g.gridConnect = occupancyGrid(5, block);
            g.gridBlock = block;
        }
        ensure(g_fused.sceneTable, sizeof(DevScene) * kMaxScenes);
        ensure(g_fused.viewTable, sizeof(ViewDesc) * kMaxScenes * kMaxViews);
        ensure(g_fused.pathScene, static_cast<size_t>(g.pathCap));
        if (!g_fused.hScenes)
            ck(cudaHostAlloc(reinterpret_cast<void**>(&g_fused.hScenes), sizeof(DevScene) * kMaxScenes,
                             cudaHostAllocDefault), "cudaHostAlloc");
        if (!g_fused.hViews)
            ck(cudaHostAlloc(reinterpret_cast<void**>(&g_fused.hViews), sizeof(ViewDesc) * kMaxScenes * kMaxViews,
                             cudaHostAllocDefault), "cudaHostAlloc");
        cudaStream_t st = g.stream;
        std::memcpy(g_fused.hScenes, table, sizeof(DevScene) * kMaxScenes);   // the previous batch frame has finished
        std::memcpy(g_fused.hViews, vd.data(), sizeof(ViewDesc) * vd.size());
        ck(cudaMemcpyAsync(g_fused.sceneTable.p, g_fused.hScenes, sizeof(DevScene) * kMaxScenes, cudaMemcpyHostToDevice,
                           st), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(g_fused.viewTable.p, g_fused.hViews, sizeof(ViewDesc) * vd.size(), cudaMemcpyHostToDevice,
                           st), "cudaMemcpyAsync");
        DevPaths P;
        std::memset(&P, 0, sizeof(P));
        P.o = g.pO.as<float4>(); P.d = g.pD.as<float4>(); P.tp = g.pTp.as<float4>(); P.L = g.pL.as<float4>();
        P.hit = g.pHit.as<float4>();
        P.queue[0] = g.q0.as<int>(); P.queue[1] = g.q1.as<int>();
        P.rayCount = g.rayCount.as<int>();
        P.shadowCount = g.shadowCount.as<int>();
        P.fetch = g.fetch.as<int>();
        P.shadowQueue = g.shadowQueue.as<int>();
        P.shOrigin = g.shOrigin.as<float4>();
        P.shDir = g.shDir.as<float4>();
        P.shContrib = g.shContrib.as<float4>();
        P.shMask = g.shMask.as<uint32_t>();
        P.slots = slots;
        P.maxDepth = depth;
        P.count = paths;
        P.errorFlags = g.errorFlags.as<unsigned int>();
        P.sortQueue = g.sortShading ? g.sortQueue.as<int>() : nullptr;
        P.sortCount = g.sortCount.as<int>();
        P.tailPaths = g.tailPaths;
        setRaySort(P, true);
        setOrder(P, true);
        P.scenes = g_fused.sceneTable.as<DevScene>();
        P.pathScene = g_fused.pathScene.as<uint8_t>();
        P.sceneCount = sceneCount;
        FrameParams f;
        std::memset(&f, 0, sizeof(f));
        f.frameIndex = g.dFrameIndex.as<uint32_t>();
        f.rrStart = rr;
        f.views = g_fused.viewTable.as<ViewDesc>();
        f.viewCount = total;
        const DevScene s = table[0];
        auto body = [&] {
            ck(cudaMemsetAsync(g.rayCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
            ck(cudaMemsetAsync(g.shadowCount.p, 0, sizeof(int) * (depth + 1), st), "cudaMemsetAsync");
            ck(cudaMemsetAsync(g.fetch.p, 0, sizeof(int) * 2 * (depth + 1), st), "cudaMemsetAsync");
            ck(cudaMemsetAsync(g.sortCount.p, 0, sizeof(int) * kSortKeys * (depth + 1), st), "cudaMemsetAsync");
            ck(cudaMemsetAsync(g.errorFlags.p, 0, 4, st), "cudaMemsetAsync");
            if (P.raySortBits > 0) ck(cudaMemsetAsync(g.binCount.p, 0, rayBinBytes(), st), "cudaMemsetAsync");
            clearOrder(P, st);
            launchGenerate(P, f, st);
            launchBounces(s, P, f, depth, block, st);
            launchTail(s, P, f, st);
            launchPresentViews(P, f, static_cast<int>(pixels64), st);
        };
        if (useGraph) {
            // the scene and view tables travel through device memory; every baked launch argument keys the capture
            std::vector<unsigned char> key;
            auto put = [&](const void* p, size_t n) {
                const unsigned char* c = static_cast<const unsigned char*>(p);
                key.insert(key.end(), c, c + n);
            };
            const int ints[9] = {depth, block, g.gridExtend, g.gridShade, g.gridConnect, g.shadeMinBlocks,
                                 static_cast<int>(pixels64), g.overlapConnect, g_scene};
            put(&P, sizeof(P)); put(&f, sizeof(f)); put(&s, sizeof(s)); put(ints, sizeof(ints));
            if (!g_fused.exec || key != g_fused.key) {
                releaseFusedGraph();
                ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                try {
                    body();
                    ck(cudaGetLastError(), "kernel launch (capture)");
                } catch (...) {
                    cudaGraph_t broken = nullptr;
                    cudaStreamEndCapture(st, &broken);
                    if (broken) cudaGraphDestroy(broken);
                    throw;
                }
                ck(cudaStreamEndCapture(st, &g_fused.graph), "cudaStreamEndCapture");
                ck(cudaGraphInstantiate(&g_fused.exec, g_fused.graph, 0), "cudaGraphInstantiate");
                g_fused.key = key;
            }
            ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
            ck(cudaGraphLaunch(g_fused.exec, st), "cudaGraphLaunch");
        } else {
            ck(cudaEventRecord(g.ev0, st), "cudaEventRecord");
            body();
        }
        ck(cudaGetLastError(), "kernel launch");
        ck(cudaEventRecord(g.ev1, st), "cudaEventRecord");
        // the frame's counters, as finishViews reads them
        g.pendDepth = depth; g.pendPaths = paths; g.pendCount = 0;
        std::vector<int> rc(static_cast<size_t>(depth + 1)), sc(static_cast<size_t>(depth + 1));
        unsigned int errFlags = 0;
        ck(cudaMemcpyAsync(rc.data(), g.rayCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(sc.data(), g.shadowCount.p, sizeof(int) * (depth + 1), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(&errFlags, g.errorFlags.p, 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(st), "frame");
        BteFrameStats S{};
        S.tailBounce = -1;
        for (int b = 0; b < depth; ++b) {
            S.extends += rc[static_cast<size_t>(b)];
            S.shadowRays += sc[static_cast<size_t>(b)];
            if (rc[static_cast<size_t>(b)] > 0) S.maxBounceReached = b;
        }
        ck(cudaEventElapsedTime(&S.msTotal, g.ev0, g.ev1), "cudaEventElapsedTime");
        // every scene: its views advance, its stats are the batch's (samples: its own)
        for (int i = 0; i < sceneCount; ++i) {
            selectScene(scenes[i]);
            g.stats = S;
            g.stats.samples = sceneSamples[static_cast<size_t>(i)];
            const BteView* sv = views + offset[static_cast<size_t>(i)];
            for (int v = 0; v < viewCounts[i]; ++v)
                g.views[static_cast<size_t>(v)].frameIndex += static_cast<uint32_t>(sv[v].samplesPerFrame);
            g.lastPaths = 0;
        }
        selectScene(home);
        if (errFlags & 1u) throw CudaError{"traversal stack overflow (BVH deeper than the traversal stack)"};
        if (errFlags & 2u) throw CudaError{"traversal met an out-of-range node or triangle index (malformed tree)"};
        if (errFlags & 4u) throw CudaError{"ordered queue compaction: a tile's wait for its predecessors gave up"};
    } catch (...) {
        selectScene(home);
        throw;
    }
    return true;
}

// One batch over several scene slots: every scene's view frame is enqueued on its own streams first, then
// each is finished in turn, so the scenes' launch sequences run side by side on the GPU.  Each scene's
// views accumulate exactly as bte_render_views would leave them; the selected slot is restored.
void renderSceneBatch(const int* scenes, const int* viewCounts, const BteView* views, int sceneCount)
{
    if (!scenes || !viewCounts || !views || sceneCount <= 0 || sceneCount > kMaxScenes)
        throw CudaError{"bte_render_scene_batch: 1..8 scenes with their view counts and views are required"};
    bool seen[kMaxScenes] = {};
    std::vector<int> offset(static_cast<size_t>(sceneCount) + 1, 0);
    for (int i = 0; i < sceneCount; ++i) {
        if (scenes[i] < 0 || scenes[i] >= kMaxScenes) throw CudaError{"bte_render_scene_batch: scene slot out of range (0..7)"};
        if (seen[scenes[i]]) throw CudaError{"bte_render_scene_batch: a scene slot appears twice"};
        seen[scenes[i]] = true;
        if (viewCounts[i] <= 0 || viewCounts[i] > kMaxViews)
            throw CudaError{"bte_render_scene_batch: each scene needs 1..64 views"};
        offset[static_cast<size_t>(i) + 1] = offset[static_cast<size_t>(i)] + viewCounts[i];
    }
    const int home = g_scene;
    if (renderSceneBatchFused(scenes, viewCounts, views, sceneCount, offset, home)) return;
    bool allGraph = true;
    for (int i = 0; i < sceneCount; ++i) {
        selectScene(scenes[i]);
        allGraph = allGraph && g.cfg.useGraph != 0;
    }
    if (allGraph) {
        renderSceneBatchGraph(scenes, viewCounts, views, sceneCount, offset, home);
        return;
    }
    std::string firstError;
    int launched = 0;
    for (; launched < sceneCount && firstError.empty(); ++launched) {
        selectScene(scenes[launched]);
        try {
            ensureInit();
            launchViews(views + offset[static_cast<size_t>(launched)], viewCounts[launched]);
        } catch (const CudaError& e) {
            firstError = e.msg;
        }
    }
    for (int i = 0; i < launched; ++i) {   // finish every enqueued frame, even after an error
        selectScene(scenes[i]);
        try {
            finishViews(views + offset[static_cast<size_t>(i)]);
        } catch (const CudaError& e) {
            if (firstError.empty()) firstError = e.msg;
        }
    }
    selectScene(home);
    if (!firstError.empty()) throw CudaError{firstError};
}

template <typename F>
int guarded(F&& fn)
{
    std::lock_guard<std::mutex> lk(g_mutex);
    try {
        ensureInit();
        return fn();
    } catch (const CudaError& e) {
        g_lastError = e.msg;
        return -1;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return -1;
    }
}

}  // namespace

void setError(const std::string& msg) { g_lastError = msg; }

}  // namespace bte

using namespace bte;

namespace {
void checkTraceFlags(const unsigned int* dFlags)
{
    unsigned int f = 0;
    ck(cudaMemcpyAsync(&f, dFlags, 4, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(g.stream), "sync");
    if (f & 1u) throw CudaError{"traversal stack overflow (BVH deeper than the traversal stack)"};
    if (f & 2u) throw CudaError{"traversal met an out-of-range node or triangle index (malformed tree)"};
}
void checkLanes(int lanes)
{
    if (lanes != 1 && lanes != 8) throw CudaError{"trace: lanesPerRay must be 1 or 8"};
    if (lanes == 8 && g.builtWidth != 8) throw CudaError{"trace: eight lanes per ray need the 8-wide tree"};
}

}  // namespace

extern "C" {

const char* bte_last_error(void) { return g_lastError.c_str(); }
int bte_version(void) { return 1; }

// src/host/scene_upload.cu:18-63
int bte_init_scene(const TriangleData* triangles, int triangleCount, const Float3* materials, int materialCount,
                   const int* triangleMaterialIds, int imageWidth, int imageHeight)
{
    (void)imageWidth; (void)imageHeight;
    return guarded([&] {
        g.tris.release(); g.materials.release(); g.triMatIds.release();
        g.bvhNodes.release(); g.wideNodes.release(); g.leafTris.release(); g.accelReady = false;
        g.triCount = triangleCount > 0 ? triangleCount : 0;
        g.materialCount = materialCount > 0 ? materialCount : 0;
        if (triangleCount > 0) upload(g.tris, triangles, sizeof(TriangleData) * triangleCount, g.stream);
        float mx = 0.0f;
        for (int i = 0; i < triangleCount; ++i) {
            const TriangleData& t = triangles[i];
            const float c[9] = {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y, t.v1.z, t.v2.x, t.v2.y, t.v2.z};
            for (float x : c) mx = std::fmax(mx, std::fabs(x));
        }
        g.sceneMaxAbs = mx;
        if (materialCount > 0) upload(g.materials, materials, sizeof(Float3) * materialCount, g.stream);
        if (triangleMaterialIds && triangleCount > 0)
            upload(g.triMatIds, triangleMaterialIds, sizeof(int) * triangleCount, g.stream);
        rebuildTriEmitter();
        ck(cudaStreamSynchronize(g.stream), "bte_init_scene");
        return 0;
    });
}

int bte_init(const TriangleData* tri, const Float3* color, int imageWidth, int imageHeight)
{
    return bte_init_scene(tri, 1, color, 1, nullptr, imageWidth, imageHeight);
}

// src/host/optix_setup.cu:298-302 (GAS build) -> LBVH
int bte_init_accel(void)
{
    return guarded([&] {
        g.bvhNodes.release(); g.wideNodes.release(); g.leafTris.release(); g.accelReady = false;
        if (!g.tris.p || g.triCount <= 0) throw CudaError{"bte_init_accel: call bte_init_scene first"};
        BvhBuildResult r;
        std::string err;
        if (buildLbvh(g.tris.as<TriangleData>(), g.triCount, g.maxLeaf, g.bvhWidth, g.bvhBuilder, g.plocRadius, g.wideCollapse, r, g.stream, err) != 0)
            throw CudaError{err};
        if (r.width == 8 && 2 * r.depth > kWideStack) {   // node + postponed-leaf groups could overflow: binary tree
            cudaFree(r.wnodes); cudaFree(r.leafTris);
            if (buildLbvh(g.tris.as<TriangleData>(), g.triCount, g.maxLeaf, 2, g.bvhBuilder, g.plocRadius, g.wideCollapse, r, g.stream, err) != 0) throw CudaError{err};
        }
        if (r.width == 8) {
            g.wideNodes.p = r.wnodes; g.wideNodes.bytes = sizeof(WideNode) * r.nodeCount;
        } else {
            g.bvhNodes.p = r.nodes; g.bvhNodes.bytes = sizeof(BvhNode) * (r.nodeCount > 0 ? r.nodeCount : 1);
        }
        g.builtWidth = r.width;
        g.builtBuilder = r.builder;
        g.accelNodes = r.nodeCount;
        g.accelDepth = r.depth;
        g.gridBlock = 0;
        g.leafTris.p = r.leafTris; g.leafTris.bytes = sizeof(float4) * 3 * static_cast<size_t>(g.triCount);
        g.rootIsLeaf = r.rootIsLeaf;
        g.rootCode = r.rootCode;
        g.msBvh = r.msBuild;
        g.accelReady = true;
        return 0;
    });
}

int bte_init_camera(const CameraData* camera)
{
    return guarded([&] {
        if (!camera) throw CudaError{"bte_init_camera: null camera"};
        g.camera = *camera;
        return 0;
    });
}

int bte_init_triangle_emission(const Float3* emission, int triangleCount)
{
    return guarded([&] {
        g.emission.release();
        if (emission && triangleCount > 0) upload(g.emission, emission, sizeof(Float3) * triangleCount, g.stream);
        ck(cudaStreamSynchronize(g.stream), "bte_init_triangle_emission");
        return 0;
    });
}

int bte_init_triangle_emitter_flags(const uint8_t* flags, int triangleCount)
{
    return guarded([&] {
        g.emitterFlags.release();
        if (flags && triangleCount > 0) upload(g.emitterFlags, flags, triangleCount, g.stream);
        ck(cudaStreamSynchronize(g.stream), "bte_init_triangle_emitter_flags");
        return 0;
    });
}

// src/host/scene_upload.cu:111-157
int bte_init_emitter_table(const EmitterData* emitters, int emitterCount, const int* emitterTriIndices,
                           int emitterTriIndexCount, const float* emitterTriCdf, int emitterTriCdfCount,
                           const float* sceneEmitterCdf)
{
    return guarded([&] {
        g.emitters.release(); g.emitterTriIndices.release(); g.emitterTriCdf.release(); g.sceneEmitterCdf.release();
        g.emitterCount = 0;
        g.hostEmitters.clear(); g.hostEmitterTriIndices.clear();
        if (emitters && emitterCount > 0 && emitterTriIndices && emitterTriIndexCount > 0 && emitterTriCdf &&
            emitterTriCdfCount > 0 && sceneEmitterCdf) {
            g.emitterCount = emitterCount;
            upload(g.emitters, emitters, sizeof(EmitterData) * emitterCount, g.stream);
            upload(g.emitterTriIndices, emitterTriIndices, sizeof(int) * emitterTriIndexCount, g.stream);
            upload(g.emitterTriCdf, emitterTriCdf, sizeof(float) * emitterTriCdfCount, g.stream);
            upload(g.sceneEmitterCdf, sceneEmitterCdf, sizeof(float) * (emitterCount + 1), g.stream);
            g.hostEmitters.assign(emitters, emitters + emitterCount);
            g.hostEmitterTriIndices.assign(emitterTriIndices, emitterTriIndices + emitterTriIndexCount);
        }
        rebuildTriEmitter();
        ck(cudaStreamSynchronize(g.stream), "bte_init_emitter_table");
        return 0;
    });
}

// src/host/scene_upload.cu:159-178
int bte_init_bsdfs(const BsdfData* bsdfs, int bsdfCount, const int* triangleBsdfIds, int triangleCount)
{
    return guarded([&] {
        g.bsdfs.release(); g.triBsdfIds.release();
        g.bsdfCount = 0;
        if (bsdfs && bsdfCount > 0 && triangleBsdfIds && triangleCount > 0) {
            for (int i = 0; i < triangleCount; ++i)
                if (triangleBsdfIds[i] < 0 || triangleBsdfIds[i] >= bsdfCount)
                    throw CudaError{"bte_init_bsdfs: triangle " + std::to_string(i) + " has BSDF id " +
                                    std::to_string(triangleBsdfIds[i]) + " outside [0, " + std::to_string(bsdfCount) + ")"};
            g.bsdfCount = bsdfCount;
            upload(g.bsdfs, bsdfs, sizeof(BsdfData) * bsdfCount, g.stream);
            upload(g.triBsdfIds, triangleBsdfIds, sizeof(int) * triangleCount, g.stream);
        }
        ck(cudaStreamSynchronize(g.stream), "bte_init_bsdfs");
        return 0;
    });
}

int bte_init_spotlights(const SpotlightData* spotlights, int spotlightCount)
{
    return guarded([&] {
        g.spots.release();
        g.spotCount = 0;
        if (spotlights && spotlightCount > 0) {
            if (spotlightCount > 30) throw CudaError{"bte_init_spotlights: at most 30 spotlights are supported"};
            g.spotCount = spotlightCount;
            upload(g.spots, spotlights, sizeof(SpotlightData) * spotlightCount, g.stream);
        }
        ck(cudaStreamSynchronize(g.stream), "bte_init_spotlights");
        return 0;
    });
}

static int initTextureSet(const uint8_t* const* pixels, const int* widths, const int* heights, int count,
                          std::vector<DeviceBuffer>& set, DeviceBuffer& table, bool isMr)
{
    return guarded([&] {
        for (auto& b : set) b.release();
        set.clear();
        table.release();
        if (!isMr) g.textureCount = 0;
        else g.hasMr = false;
        if (!pixels || count <= 0) return 0;
        set.resize(static_cast<size_t>(count));
        std::vector<TexRef> refs(static_cast<size_t>(count), TexRef{nullptr, 0, 0});
        for (int i = 0; i < count; ++i) {
            if (!pixels[i]) continue;
            if (widths[i] <= 0 || heights[i] <= 0) throw CudaError{"texture with non-positive size"};
            upload(set[static_cast<size_t>(i)], pixels[i], static_cast<size_t>(widths[i]) * heights[i] * 4, g.stream);
            refs[static_cast<size_t>(i)] = TexRef{set[static_cast<size_t>(i)].as<uchar4>(), widths[i], heights[i]};
        }
        upload(table, refs.data(), refs.size() * sizeof(TexRef), g.stream);
        ck(cudaStreamSynchronize(g.stream), "texture upload");
        if (!isMr) g.textureCount = count;
        else g.hasMr = true;
        return 0;
    });
}

// src/host/scene_upload.cu:213-293
int bte_init_textures(const uint8_t* const* pixels, const int* widths, const int* heights, int count)
{
    return initTextureSet(pixels, widths, heights, count, g.tex, g.texTable, false);
}
int bte_init_mr_textures(const uint8_t* const* pixels, const int* widths, const int* heights, int count)
{
    return initTextureSet(pixels, widths, heights, count, g.texMr, g.texTableMr, true);
}

// src/host/scene_upload.cu:390-484
int bte_init_env_map(const float* rgba, int width, int height, float intensity, float rotationDeg)
{
    return guarded([&] {
        for (DeviceBuffer* b : {&g.envTexels, &g.envMarginal, &g.envConditional, &g.envRowProb, &g.envRowAlias,
                                &g.envColProb, &g.envColAlias, &g.envPixelPdf})
            b->release();
        g.hasEnv = false;
        g.envW = g.envH = 0;
        g.envTotalPowerF = 0.0f;
        g.envTotalPowerD = 0.0;
        if (!rgba || width <= 0 || height <= 0) return 0;
        const size_t n = static_cast<size_t>(width) * height;
        upload(g.envTexels, rgba, n * 16, g.stream);
        ensure(g.envMarginal, sizeof(float) * (height + 1));
        ensure(g.envConditional, sizeof(float) * static_cast<size_t>(height) * (width + 1));
        ensure(g.envRowProb, sizeof(float) * height);
        ensure(g.envRowAlias, sizeof(int) * height);
        ensure(g.envColProb, sizeof(float) * n);
        ensure(g.envColAlias, sizeof(int) * n);
        ensure(g.envPixelPdf, sizeof(float) * n);
        // theta at each row centre and its sine, evaluated as the reference's host loop does
        const float PI = 3.14159265358979323846f;
        std::vector<float> sinT(static_cast<size_t>(height));
        for (int iy = 0; iy < height; ++iy) {
            const float theta = PI * (static_cast<float>(iy) + 0.5f) / static_cast<float>(height);
            sinT[static_cast<size_t>(iy)] = std::sin(theta);
        }
        std::string err;
        if (buildEnvCdf(g.envTexels.as<float4>(), width, height, sinT.data(), g.envMarginal.as<float>(),
                        g.envConditional.as<float>(), g.stream, err) != 0)
            throw CudaError{err};
        if (buildEnvAlias(g.envTexels.as<float4>(), width, height, g.envRowProb.as<float>(), g.envRowAlias.as<int>(),
                          g.envColProb.as<float>(), g.envColAlias.as<int>(), g.envPixelPdf.as<float>(), &g.envTotalPowerD,
                          g.stream, err) != 0)
            throw CudaError{err};
        ck(cudaMemcpyAsync(&g.envTotalPowerF, g.envMarginal.as<float>() + height, sizeof(float), cudaMemcpyDeviceToHost,
                           g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        g.envW = width; g.envH = height;
        g.envIntensity = intensity;
        g.envRotation = rotationDeg * (PI / 180.0f);
        g.hasEnv = true;
        return 0;
    });
}

int bte_set_output_buffer(uint32_t* deviceRGBA8)
{
    return guarded([&] { g.extFramebuffer = deviceRGBA8; return 0; });
}

// src/render_kernel.cu:40-56
int bte_reset_accumulation(int imageWidth, int imageHeight)
{
    return guarded([&] {
        if (imageWidth <= 0 || imageHeight <= 0) throw CudaError{"bte_reset_accumulation: size must be positive"};
        ensureAccum(imageWidth, imageHeight);
        return 0;
    });
}

// src/render_kernel.cu:58-144
int bte_render(int imageWidth, int imageHeight)
{
    return guarded([&] {
        if (g.sceneChanged) {   // src/main.cpp:947-952: reset before the frame that follows a change
            ensureAccum(imageWidth, imageHeight);
            g.sceneChanged = false;
        }
        renderFrame(imageWidth, imageHeight);
        return 0;
    });
}

int bte_mark_scene_changed(void)
{
    return guarded([&] { g.sceneChanged = true; return 0; });
}

int bte_get_framebuffer_size(int* width, int* height)
{
    return guarded([&] {
        if (!g.framebuffer.p) throw CudaError{"bte_get_framebuffer_size: nothing rendered"};
        if (width) *width = g.accumW;
        if (height) *height = g.accumH;
        return 0;
    });
}

// render_kernel.h:187 (cudaToggleDenoiser): returns the new state.  Turning
// it on needs denoiser weights (bte_denoiser_set_params / bte_denoiser_init)
// and switches the albedo / normal features on; each frame then presents the
// denoised accumulation.  Plain accumulation stays the buffer of record.
int bte_render_views(const BteView* views, int count)
{
    return guarded([&] {
        renderViews(views, count);
        return 0;
    });
}

int bte_read_view_accum(int view, float* hostRGB, double* hostRGBSum)
{
    return guarded([&] {
        if (view < 0 || view >= static_cast<int>(g.views.size()) || !g.views[static_cast<size_t>(view)].accum.p)
            throw CudaError{"bte_read_view_accum: no such view (bte_render_views)"};
        const Renderer::ViewState& v = g.views[static_cast<size_t>(view)];
        if (hostRGB)
            ck(cudaMemcpyAsync(hostRGB, v.accum.p, v.accum.bytes, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        if (hostRGBSum)
            ck(cudaMemcpyAsync(hostRGBSum, v.accumD.p, v.accumD.bytes, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

int bte_reset_views(void)
{
    return guarded([&] {
        for (auto& v : g.views) { v.accum.release(); v.accumD.release(); v.fb.release(); }
        g.views.clear();
        return 0;
    });
}

int bte_select_scene(int scene)
{
    return guarded([&] {
        selectScene(scene);
        ensureInit();
        return 0;
    });
}

int bte_get_selected_scene(int* scene)
{
    return guarded([&] {
        if (!scene) throw CudaError{"bte_get_selected_scene: null pointer"};
        *scene = g_scene;
        return 0;
    });
}

int bte_set_batch_mode(int mode)
{
    return guarded([&] {
        if (mode != 0 && mode != 1) throw CudaError{"bte_set_batch_mode: mode must be 0 or 1"};
        g_batchMode = mode;
        return 0;
    });
}

int bte_get_batch_mode(int* mode)
{
    return guarded([&] {
        if (!mode) throw CudaError{"bte_get_batch_mode: null pointer"};
        *mode = g_batchMode;
        return 0;
    });
}

int bte_render_scene_batch(const int* scenes, const int* viewCounts, const BteView* views, int sceneCount)
{
    return guarded([&] {
        renderSceneBatch(scenes, viewCounts, views, sceneCount);
        return 0;
    });
}

int bte_toggle_denoiser(void)
{
    return guarded([&]() -> int {
        if (!g.denoiser && !dn::denoiserReady())
            throw CudaError{"bte_toggle_denoiser: no denoiser weights (bte_denoiser_set_params or bte_denoiser_init)"};
        g.denoiser = !g.denoiser;
        if (g.denoiser && !g.aovEnabled) {
            g.aovEnabled = true;
            if (g.accumW > 0) ensureAccum(g.accumW, g.accumH);   // features and radiance restart together
        }
        return g.denoiser ? 1 : 0;
    });
}

// include/optix_launch_params.h:34-86: the reference fills this block before every launch
// (render_kernel.cu:58-143, wavefront_host.cu:122-148); here it is filled on request from the current state.
int bte_get_launch_params(LaunchParams* out)
{
    return guarded([&] {
        if (!out) throw CudaError{"bte_get_launch_params: null pointer"};
        LaunchParams p;
        std::memset(&p, 0, sizeof(p));
        p.framebuffer = g.framebuffer.as<uint32_t>();
        p.accumBuffer = g.accum.as<Float3>();
        p.width = g.accumW;
        p.height = g.accumH;
        p.launchOffsetY = 0;
        p.frameIndex = g.frameIndex;
        p.camera = g.camera;
        const void* tree = g.builtWidth == 8 ? g.wideNodes.p : g.bvhNodes.p;
        p.handle = g.accelReady ? static_cast<uint64_t>(reinterpret_cast<uintptr_t>(tree)) : 0u;
        p.triangles = g.tris.as<TriangleData>();
        p.triangleCount = g.triCount;
        p.bsdfs = g.bsdfs.as<BsdfData>();
        p.bsdfCount = g.bsdfCount;
        p.triangleBsdfIds = g.triBsdfIds.as<int>();
        p.triangleMaterialIds = g.triMatIds.as<int>();
        p.triangleEmitterFlags = g.emitterFlags.as<uint8_t>();
        p.triangleEmission = g.emission.as<Float3>();
        p.emitters = g.emitters.as<EmitterData>();
        p.emitterCount = g.emitterCount;
        p.emitterTriIndices = g.emitterTriIndices.as<int>();
        p.emitterTriCdf = g.emitterTriCdf.as<float>();
        p.sceneEmitterCdf = g.sceneEmitterCdf.as<float>();
        p.spotlights = g.spots.as<SpotlightData>();
        p.spotlightCount = g.spotCount;
        p.texObjects = nullptr;
        p.texObjectsMr = nullptr;
        p.textureCount = g.textureCount;
        if (g.hasEnv) {
            p.envMap.texObj = 0;
            p.envMap.width = g.envW;
            p.envMap.height = g.envH;
            p.envMap.intensity = g.envIntensity;
            p.envMap.rotationRadians = g.envRotation;
            p.envMap.marginalCdf = g.envMarginal.as<float>();
            p.envMap.conditionalCdf = g.envConditional.as<float>();
            p.envMap.totalPower = g.envTotalPowerF;
        }
        p.hasEnvMap = g.hasEnv;
        p.wf.rayQueue = g.q0.as<int>();
        p.wf.rayQueueNext = g.q1.as<int>();
        p.wf.rayCount = g.rayCount.as<int>();
        p.wf.rayCountNext = g.rayCount.p ? g.rayCount.as<int>() + 1 : nullptr;
        p.wf.shadowCount = g.shadowCount.as<int>();
        p.wf.maxPaths = g.lastPaths;
        p.wf.maxShadows = g.lastPaths * g.lastSlots;
        *out = p;
        return 0;
    });
}

int bte_read_denoised(float* hostRGB)
{
    return guarded([&] {
        if (!g.denoised.p) throw CudaError{"bte_read_denoised: no denoised frame (bte_toggle_denoiser, then bte_render)"};
        ck(cudaMemcpyAsync(hostRGB, g.denoised.p, g.denoised.bytes, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

// src/render_kernel.cu:171-183
int bte_set_render_mode(int mode)
{
    return guarded([&] {
        if (mode != BTE_RENDER_MEGAKERNEL && mode != BTE_RENDER_WAVEFRONT) throw CudaError{"bte_set_render_mode: bad mode"};
        if (mode != g.renderMode) {
            g.renderMode = mode;
            if (g.accumW > 0) ensureAccum(g.accumW, g.accumH);
        }
        return 0;
    });
}
int bte_get_render_mode(void) { return g.renderMode; }

// src/render_kernel.cu:146-168
int bte_cleanup(void)
{
    return guarded([&] {
        for (DeviceBuffer* b : {&g.tris, &g.materials, &g.triMatIds, &g.emission, &g.emitterFlags, &g.triEmitter,
                                &g.emitters, &g.emitterTriIndices, &g.emitterTriCdf, &g.sceneEmitterCdf, &g.bsdfs,
                                &g.triBsdfIds, &g.spots, &g.texTable, &g.texTableMr, &g.envTexels, &g.envMarginal,
                                &g.envConditional, &g.envRowProb, &g.envRowAlias, &g.envColProb, &g.envColAlias,
                                &g.envPixelPdf, &g.bvhNodes, &g.wideNodes, &g.leafTris, &g.accum, &g.accumD, &g.framebuffer,
                                &g.aovAccum, &g.denoised})
            b->release();
        for (auto& b : g.tex) b.release();
        for (auto& b : g.texMr) b.release();
        g.tex.clear(); g.texMr.clear();
        releaseGraph();
        releaseWavefront();
        g.triCount = g.materialCount = g.emitterCount = g.bsdfCount = g.spotCount = g.textureCount = 0;
        g.hasEnv = false; g.hasMr = false; g.accelReady = false;
        g.accumW = g.accumH = 0; g.frameIndex = 0; g.extFramebuffer = nullptr;
        g.hostEmitters.clear(); g.hostEmitterTriIndices.clear();
        return 0;
    });
}

int bte_set_render_config(const BteRenderConfig* cfg)
{
    return guarded([&] {
        if (!cfg) throw CudaError{"bte_set_render_config: null config"};
        if (cfg->samplesPerFrame < 1 || cfg->maxDepth < 1 || cfg->maxDepth > 1024)
            throw CudaError{"bte_set_render_config: samplesPerFrame >= 1 and 1 <= maxDepth <= 1024 required"};
        if (cfg->envSampling != BTE_ENV_SAMPLING_CDF && cfg->envSampling != BTE_ENV_SAMPLING_ALIAS)
            throw CudaError{"bte_set_render_config: bad envSampling"};
        if (cfg->blockSize != 0 && (cfg->blockSize < 32 || cfg->blockSize > 256 || cfg->blockSize % 32 != 0))
            throw CudaError{"bte_set_render_config: blockSize must be 0 or a multiple of 32 in [32, 256]"};
        g.cfg = *cfg;
        return 0;
    });
}
int bte_get_render_config(BteRenderConfig* cfg)
{
    return guarded([&] { if (cfg) *cfg = g.cfg; return 0; });
}
int bte_get_frame_stats(BteFrameStats* out)
{
    return guarded([&] { if (out) *out = g.stats; return 0; });
}
int bte_set_stage_timing(int enabled)
{
    return guarded([&] { g.stageTiming = enabled != 0; return 0; });
}
int bte_get_frame_index(uint32_t* out)
{
    return guarded([&] { if (out) *out = g.frameIndex; return 0; });
}
int bte_set_frame_index(uint32_t frameIndex)
{
    return guarded([&] { g.frameIndex = frameIndex; return 0; });
}
int bte_set_tuning(const BteTuning* t)
{
    return guarded([&] {
        if (!t) throw CudaError{"bte_set_tuning: null tuning"};
        if (t->bvhWidth != 2 && t->bvhWidth != 8) throw CudaError{"bte_set_tuning: bvhWidth must be 2 or 8"};
        const int leafMax = t->bvhWidth == 8 ? kWideLeafMax : kMaxLeafTris;
        if (t->maxLeafTriangles < 1 || t->maxLeafTriangles > leafMax)
            throw CudaError{"bte_set_tuning: maxLeafTriangles must be in [1, 64] (binary) or [1, 3] (8-wide)"};
        if (t->shadeMinBlocks < 2 || t->shadeMinBlocks > 4) throw CudaError{"bte_set_tuning: shadeMinBlocks must be 2, 3 or 4"};
        if (t->postponePercent < 0 || t->postponePercent > 100) throw CudaError{"bte_set_tuning: postponePercent in [0, 100]"};
        if (t->sortShading != 0 && t->sortShading != 1) throw CudaError{"bte_set_tuning: sortShading must be 0 or 1"};
        if (t->tailPaths < 0) throw CudaError{"bte_set_tuning: tailPaths must be >= 0"};
        if (t->bvhBuilder != 0 && t->bvhBuilder != 1) throw CudaError{"bte_set_tuning: bvhBuilder must be 0 or 1"};
        if (t->plocRadius < 1 || t->plocRadius > kPlocMaxRadius) throw CudaError{"bte_set_tuning: plocRadius in [1, 32]"};
        if (t->overlapConnect != 0 && t->overlapConnect != 1) throw CudaError{"bte_set_tuning: overlapConnect must be 0 or 1"};
        if (t->wideCollapse != 0 && t->wideCollapse != 1) throw CudaError{"bte_set_tuning: wideCollapse must be 0 or 1"};
        if (t->raySortBits < 0 || t->raySortBits > 4) throw CudaError{"bte_set_tuning: raySortBits in [0, 4]"};
        if (t->raySortBounces < 1 || t->raySortBounces > 64) throw CudaError{"bte_set_tuning: raySortBounces in [1, 64]"};
        if (t->leafTestsPerStep < 0 || t->leafTestsPerStep > 24)
            throw CudaError{"bte_set_tuning: leafTestsPerStep in [0, 24]"};
        if (t->orderBounces < 0 || t->orderBounces > 64) throw CudaError{"bte_set_tuning: orderBounces in [0, 64]"};
        g.bvhWidth = t->bvhWidth;
        g.maxLeaf = t->maxLeafTriangles;
        g.shadeMinBlocks = t->shadeMinBlocks;
        g.postponePct = t->postponePercent;
        g.sortShading = t->sortShading;
        g.tailPaths = t->tailPaths;
        g.bvhBuilder = t->bvhBuilder;
        g.plocRadius = t->plocRadius;
        g.overlapConnect = t->overlapConnect;
        g.wideCollapse = t->wideCollapse;
        g.raySortBits = t->raySortBits;
        g.raySortBounces = t->raySortBounces;
        g.leafTestsPerStep = t->leafTestsPerStep;
        g.orderBounces = t->orderBounces;
        g.gridBlock = 0;   // recompute persistent grids
        return 0;
    });
}

int bte_get_tuning(BteTuning* t)
{
    return guarded([&] {
        if (!t) throw CudaError{"bte_get_tuning: null tuning"};
        t->bvhWidth = g.bvhWidth;
        t->maxLeafTriangles = g.maxLeaf;
        t->shadeMinBlocks = g.shadeMinBlocks;
        t->postponePercent = g.postponePct;
        t->sortShading = g.sortShading;
        t->tailPaths = g.tailPaths;
        t->bvhBuilder = g.bvhBuilder;
        t->plocRadius = g.plocRadius;
        t->overlapConnect = g.overlapConnect;
        t->wideCollapse = g.wideCollapse;
        t->raySortBits = g.raySortBits;
        t->raySortBounces = g.raySortBounces;
        t->leafTestsPerStep = g.leafTestsPerStep;
        t->orderBounces = g.orderBounces;
        return 0;
    });
}

int bte_get_accel_builder(int* builder)
{
    return guarded([&] {
        if (!g.accelReady) throw CudaError{"bte_get_accel_builder: no acceleration structure (bte_init_accel)"};
        if (!builder) throw CudaError{"bte_get_accel_builder: null builder"};
        *builder = g.builtBuilder;
        return 0;
    });
}

int bte_get_accel_info(int* width, int* nodeCount, int* depth, float* msBuild)
{
    return guarded([&] {
        if (!g.accelReady) throw CudaError{"bte_get_accel_info: no acceleration structure (bte_init_accel)"};
        if (width) *width = g.builtWidth;
        if (nodeCount) *nodeCount = g.accelNodes;
        if (depth) *depth = g.accelDepth;
        if (msBuild) *msBuild = g.msBvh;
        return 0;
    });
}

int bte_set_aov(int enabled)
{
    return guarded([&] {
        g.aovEnabled = enabled != 0 || g.denoiser;   // the denoiser keeps its features
        if (!g.aovEnabled) { g.aovAlbedo.release(); g.aovNormal.release(); g.aovAccum.release(); }
        return 0;
    });
}

int bte_read_aov(float* hostAlbedoNormal)
{
    return guarded([&] {
        if (!g.aovEnabled || !g.aovAccum.p) throw CudaError{"bte_read_aov: features not enabled (bte_set_aov) or not rendered"};
        ck(cudaMemcpyAsync(hostAlbedoNormal, g.aovAccum.p, g.aovAccum.bytes, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

int bte_set_hit_log(int enabled)
{
    return guarded([&] { g.hitLogEnabled = enabled != 0; if (!g.hitLogEnabled) g.hitLog.release(); return 0; });
}

int bte_read_framebuffer(uint32_t* host)
{
    return guarded([&] {
        if (!g.framebuffer.p) throw CudaError{"bte_read_framebuffer: nothing rendered"};
        ck(cudaMemcpyAsync(host, g.framebuffer.p, static_cast<size_t>(g.accumW) * g.accumH * 4, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}
int bte_read_accum(float* host)
{
    return guarded([&] {
        if (!g.accum.p) throw CudaError{"bte_read_accum: nothing rendered"};
        ck(cudaMemcpyAsync(host, g.accum.p, static_cast<size_t>(g.accumW) * g.accumH * 12, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}
int bte_read_accum_f64(double* host)
{
    return guarded([&] {
        if (!g.accumD.p) throw CudaError{"bte_read_accum_f64: nothing rendered"};
        ck(cudaMemcpyAsync(host, g.accumD.p, static_cast<size_t>(g.accumW) * g.accumH * 24, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}
int bte_read_sample_radiance(float* host, int count)
{
    return guarded([&] {
        if (count < 0 || count > g.lastPaths) throw CudaError{"bte_read_sample_radiance: count out of range"};
        std::vector<float4> tmp(static_cast<size_t>(count));
        ck(cudaMemcpyAsync(tmp.data(), g.pL.p, sizeof(float4) * count, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        for (int i = 0; i < count; ++i) {
            host[3 * i] = tmp[static_cast<size_t>(i)].x;
            host[3 * i + 1] = tmp[static_cast<size_t>(i)].y;
            host[3 * i + 2] = tmp[static_cast<size_t>(i)].z;
        }
        return 0;
    });
}
int bte_read_hit_log(int* host, int count)
{
    return guarded([&] {
        if (!g.hitLog.p) throw CudaError{"bte_read_hit_log: enable with bte_set_hit_log before rendering"};
        if (count < 0 || static_cast<long long>(count) > static_cast<long long>(g.lastPaths) * g.lastDepth)
            throw CudaError{"bte_read_hit_log: count out of range"};
        ck(cudaMemcpyAsync(host, g.hitLog.p, sizeof(int) * count, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

}  // extern "C"

// ---- debug / parity entry points ----
namespace {
template <typename T>
struct Tmp {
    T* p = nullptr;
    explicit Tmp(size_t n) { ck(cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)), "cudaMalloc"); }
    ~Tmp() { cudaFree(p); }
};
}  // namespace

extern "C" {

int bte_trace_closest_lanes(const float* rays, int n, int lanesPerRay, int* outTri, float* outTuv)
{
    return guarded([&] {
        if (n <= 0) return 0;
        if (!g.accelReady) throw CudaError{"bte_trace_closest: no acceleration structure"};
        checkLanes(lanesPerRay);
        Tmp<float> dr(6 * static_cast<size_t>(n)), dt(3 * static_cast<size_t>(n));
        Tmp<int> di(n);
        Tmp<unsigned int> de(1);
        ck(cudaMemcpyAsync(dr.p, rays, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        ck(cudaMemsetAsync(de.p, 0, 4, g.stream), "cudaMemsetAsync");
        launchTraceClosestRays(makeDevScene(), dr.p, n, di.p, dt.p, de.p, lanesPerRay, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "trace");
        ck(cudaMemcpyAsync(outTri, di.p, sizeof(int) * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        ck(cudaMemcpyAsync(outTuv, dt.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        checkTraceFlags(de.p);
        return 0;
    });
}

int bte_trace_occluded_lanes(const float* rays, const float* tmax, int n, int lanesPerRay, uint8_t* outOccluded)
{
    return guarded([&] {
        if (n <= 0) return 0;
        if (!g.accelReady) throw CudaError{"bte_trace_occluded: no acceleration structure"};
        checkLanes(lanesPerRay);
        Tmp<float> dr(6 * static_cast<size_t>(n)), dm(n);
        Tmp<uint8_t> dout(n);
        Tmp<unsigned int> de(1);
        ck(cudaMemcpyAsync(dr.p, rays, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(dm.p, tmax, sizeof(float) * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        ck(cudaMemsetAsync(de.p, 0, 4, g.stream), "cudaMemsetAsync");
        launchTraceOccludedRays(makeDevScene(), dr.p, dm.p, n, dout.p, de.p, lanesPerRay, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "trace");
        ck(cudaMemcpyAsync(outOccluded, dout.p, n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        checkTraceFlags(de.p);
        return 0;
    });
}

int bte_debug_lbvh_order(const TriangleData* triangles, int n, uint64_t* mortonKeys, int* sortedOrder)
{
    return guarded([&] {
        if (!triangles || !mortonKeys || !sortedOrder || n <= 0) throw CudaError{"bte_debug_lbvh_order: bad arguments"};
        ensureInit();
        std::string err;
        if (lbvhMortonOrder(triangles, n, reinterpret_cast<unsigned long long*>(mortonKeys), sortedOrder, err) != 0)
            throw CudaError{err};
        return 0;
    });
}

int bte_trace_closest(const float* rays, int n, int* outTri, float* outTuv)
{
    return bte_trace_closest_lanes(rays, n, 1, outTri, outTuv);
}

int bte_trace_occluded(const float* rays, const float* tmax, int n, uint8_t* outOccluded)
{
    return bte_trace_occluded_lanes(rays, tmax, n, 1, outOccluded);
}

int bte_env_query(int op, const float* in, int n, float* out)
{
    return guarded([&] {
        if (n <= 0) return 0;
        if (!g.hasEnv) throw CudaError{"bte_env_query: no environment map"};
        const size_t inN = (op == 2 ? 2 : 3) * static_cast<size_t>(n);
        const size_t outN = (op == 0 ? 3 : (op == 1 ? 1 : 7)) * static_cast<size_t>(n);
        Tmp<float> di(inN), dout(outN);
        ck(cudaMemcpyAsync(di.p, in, sizeof(float) * inN, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        launchEnvQuery(makeDevScene(), op, di.p, n, dout.p, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "env query");
        ck(cudaMemcpyAsync(out, dout.p, sizeof(float) * outN, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

int bte_env_tables(float* marginal, float* conditional, float* totalPower)
{
    return guarded([&] {
        if (!g.hasEnv) throw CudaError{"bte_env_tables: no environment map"};
        if (marginal) ck(cudaMemcpyAsync(marginal, g.envMarginal.p, sizeof(float) * (g.envH + 1), cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        if (conditional)
            ck(cudaMemcpyAsync(conditional, g.envConditional.p, sizeof(float) * static_cast<size_t>(g.envH) * (g.envW + 1),
                               cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(g.stream), "sync");
        if (totalPower) *totalPower = g.envTotalPowerF;
        return 0;
    });
}

int bte_env_alias_tables(float* rowProb, int* rowIdx, float* colProb, int* colIdx, float* pixelPdf)
{
    return guarded([&] {
        if (!g.hasEnv) throw CudaError{"bte_env_alias_tables: no environment map"};
        const size_t n = static_cast<size_t>(g.envW) * g.envH;
        if (rowProb) ck(cudaMemcpyAsync(rowProb, g.envRowProb.p, sizeof(float) * g.envH, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        if (rowIdx) ck(cudaMemcpyAsync(rowIdx, g.envRowAlias.p, sizeof(int) * g.envH, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        if (colProb) ck(cudaMemcpyAsync(colProb, g.envColProb.p, sizeof(float) * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        if (colIdx) ck(cudaMemcpyAsync(colIdx, g.envColAlias.p, sizeof(int) * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        if (pixelPdf) ck(cudaMemcpyAsync(pixelPdf, g.envPixelPdf.p, sizeof(float) * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

int bte_math_eval(int fn, const float* a, const float* b, float* out, int n)
{
    return guarded([&] {
        if (n <= 0) return 0;
        Tmp<float> da(n), db(n), dout(n);
        ck(cudaMemcpyAsync(da.p, a, sizeof(float) * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        if (b) ck(cudaMemcpyAsync(db.p, b, sizeof(float) * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        else ck(cudaMemsetAsync(db.p, 0, sizeof(float) * n, g.stream), "cudaMemsetAsync");
        launchMathEval(fn, da.p, db.p, dout.p, n, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "math");
        ck(cudaMemcpyAsync(out, dout.p, sizeof(float) * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

int bte_bsdf_query(const BsdfData* bsdf, int op, const float* wi, const float* woOrU, int n, float* out)
{
    return guarded([&] {
        if (n <= 0) return 0;
        if (!bsdf || op < 0 || op > 2) throw CudaError{"bte_bsdf_query: bad arguments"};
        const size_t outN = (op == 0 ? 3 : (op == 1 ? 1 : 8)) * static_cast<size_t>(n);
        Tmp<float> dwi(3 * static_cast<size_t>(n)), dx(3 * static_cast<size_t>(n)), dout(outN);
        ck(cudaMemcpyAsync(dwi.p, wi, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(dx.p, woOrU, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        launchBsdfQuery(*bsdf, op, dwi.p, dx.p, n, dout.p, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "bsdf");
        ck(cudaMemcpyAsync(out, dout.p, sizeof(float) * outN, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

// Hardware tex2D with the reference's env-map texture settings
// (src/host/scene_upload.cu:406-420) against the library's software filter.
int bte_tex_hw_vs_sw(const float* texels, int w, int h, int wrapV, const float* uv, int n, float* outHw, float* outSw)
{
    return guarded([&] {
        if (n <= 0 || w <= 0 || h <= 0) return 0;
        cudaArray_t arr = nullptr;
        cudaTextureObject_t tex = 0;
        const cudaChannelFormatDesc desc = cudaCreateChannelDesc<float4>();
        ck(cudaMallocArray(&arr, &desc, w, h), "cudaMallocArray");
        struct Guard {
            cudaArray_t a; cudaTextureObject_t* t;
            ~Guard() { if (*t) cudaDestroyTextureObject(*t); cudaFreeArray(a); }
        } guard{arr, &tex};
        ck(cudaMemcpy2DToArrayAsync(arr, 0, 0, texels, static_cast<size_t>(w) * 16, static_cast<size_t>(w) * 16, h,
                                    cudaMemcpyHostToDevice, g.stream), "cudaMemcpy2DToArrayAsync");
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = wrapV ? cudaAddressModeWrap : cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        ck(cudaCreateTextureObject(&tex, &rd, &td, nullptr), "cudaCreateTextureObject");
        Tmp<float4> dt(static_cast<size_t>(w) * h);
        Tmp<float> duv(2 * static_cast<size_t>(n)), dhw(4 * static_cast<size_t>(n)), dsw(4 * static_cast<size_t>(n));
        ck(cudaMemcpyAsync(dt.p, texels, sizeof(float4) * w * h, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        ck(cudaMemcpyAsync(duv.p, uv, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, g.stream), "cudaMemcpyAsync");
        launchTexCompare(tex, dt.p, w, h, wrapV, duv.p, n, dhw.p, dsw.p, g.stream);
        ck(cudaGetLastError(), "launch");
        ck(cudaStreamSynchronize(g.stream), "tex compare");
        ck(cudaMemcpyAsync(outHw, dhw.p, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        ck(cudaMemcpyAsync(outSw, dsw.p, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost, g.stream), "cudaMemcpyAsync"); ck(cudaStreamSynchronize(g.stream), "sync");
        return 0;
    });
}

}  // extern "C"
