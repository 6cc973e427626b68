// bte_types.cuh -- device-side data layout of the renderer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/bte/render_api.h"

#define BTE_DI __device__ __forceinline__

namespace bte {

struct V3 { float x, y, z; };

struct TexRef { const uchar4* pixels; int w, h; };

// Environment map: float4 texels (wrap u, clamp v) plus either the
// reference's marginal/conditional CDF or the two-level alias tables.
struct DevEnv {
    const float4* texels;
    int w, h;
    float intensity, rotation;        // rotation in radians
    float totalPower;
    int sampling;                     // BTE_ENV_SAMPLING_*
    const float* marginal;            // [h+1]
    const float* conditional;         // [h*(w+1)]
    const float* rowProb; const int* rowAlias;   // [h]
    const float* colProb; const int* colAlias;   // [h*w]
    const float* pixelPdf;                        // [h*w]
};

// BVH2 node: the two children's boxes side by side (one 64-byte fetch tests
// both).  A child index c >= 0 is an inner node; c < 0 is a leaf holding
// triangles [start, start+count) of the leaf-ordered triangle array with
// ~c = start | (count-1) << 25.
struct BvhNode {
    float4 lxy;    // child0: lo.x, hi.x, lo.y, hi.y
    float4 rxy;    // child1: lo.x, hi.x, lo.y, hi.y
    float4 z;      // child0 lo.z, hi.z, child1 lo.z, hi.z
    int4 child;    // child0, child1, unused, unused
};
constexpr int kLeafCountShift = 25;
constexpr int kLeafStartMask = (1 << kLeafCountShift) - 1;
constexpr int kMaxLeafTris = 64;

// 8-wide node with 8-bit quantised child boxes (80 bytes, five 16-byte
// loads).  Child box coordinate = fma(q, 2^(e-127), p) per axis, which the
// build makes contain the child's exact box.  Internal children are stored
// consecutively from childBase in slot order (child of slot s =
// childBase + popc(imask & ((1<<s)-1))); a leaf slot's meta byte is
// offset | count << 5 into the node's triangles starting at triBase; a slot
// with neither is empty.  Slots are assigned so that a ray of direction
// octant q visits them in increasing (slot ^ q) order, near side first.
struct WideNode {
    float px, py, pz;
    uint32_t expImask;            // ex | ey << 8 | ez << 16 | imask << 24
    int childBase;
    int triBase;
    uint32_t meta[2];
    uint32_t qlox[2], qloy[2], qloz[2], qhix[2], qhiy[2], qhiz[2];
};
static_assert(sizeof(WideNode) == 80, "WideNode is five 16-byte words");
constexpr int kWideLeafMax = 3;
constexpr int kSortKeys = 6;
constexpr int kWideStack = 64;    // traversal stack entries; trees deeper than half of it use the binary tree
constexpr int kTraversalStack = 96;   // binary-tree traversal stack entries; deeper PLOC trees fall back to LBVH
constexpr int kPlocMaxRadius = 32;   // PLOC neighbour search radius limit (positions each side)

struct DevScene {
    // geometry
    const TriangleData* tris;         // reference AoS, original triangle order
    int triCount;
    const float4* leafTris;           // [triCount*3] v0.xyz|origIndex, v1.xyz, v2.xyz in leaf order of the tree in use
    const BvhNode* nodes;             // root = node 0 (triCount >= 2) or a single-leaf root
    const WideNode* wnodes;           // 8-wide tree (root = node 0) when bvhWidth == 8
    int bvhWidth;                     // 2 or 8
    int wideNodeCount;
    int postponePct;                  // leaf-test postponing threshold of the 8-wide walk (percent of lanes)
    int leafTestsPerStep;             // 8-wide walk: triangle tests per walk step (0: all of the node's)
    int rootIsLeaf;                   // the whole scene is one leaf
    int rootCode;                     // its leaf code
    float sceneMaxAbs;                // max |coordinate| over all vertices (traversal error bound)
    // materials
    const BsdfData* bsdfs;
    const int* triBsdfIds;
    const int* triMaterialIds;
    const TexRef* texTable; const TexRef* texTableMr; int textureCount;
    // emission
    const uint8_t* emitterFlags;
    const Float3* emission;
    const int* triEmitter;            // triangle -> first emitter containing it, or -1
    const EmitterData* emitters; int emitterCount;
    const int* emitterTriIndices;
    const float* emitterTriCdf;
    const float* sceneEmitterCdf;
    const SpotlightData* spots; int spotCount;
    int hasEnv;
    DevEnv env;
};

// Per-path wavefront state (structure of arrays, 16-byte records).
struct DevPaths {
    float4* o;        // ray origin xyz | rng state (bits)
    float4* d;        // ray direction xyz | eta
    float4* tp;       // throughput xyz | brdfPdf of the last scatter
    float4* L;        // radiance xyz | bounce (bits 0-15) | specular (bit 16)
    float4* hit;      // t, u, v | triangle index (bits; -1 miss)
    int* queue[2];    // ping-pong ray queues of path indices
    int* rayCount;    // [maxDepth+1] active paths per bounce
    int* shadowCount; // [maxDepth] shadow rays per bounce
    int* fetch;       // [2*(maxDepth+1)] ray-fetch counters of the extend / connect launches
    int* shadowQueue; // entries path*slots + slot
    float4* shOrigin; // [paths] hit point of the NEE rays of the current bounce
    float4* shDir;    // [paths*slots] direction | tmax
    float4* shContrib;// [paths*slots] contribution | unused
    uint32_t* shMask; // [paths] bit s: slot s visible and not yet added
    int* hitLog;      // optional [paths*maxDepth]
    float4* aovAlbedo;// optional [paths] feature albedo (denoiser feature)
    float4* aovNormal;// optional [paths] feature shading normal (denoiser feature)
    int slots;        // 1 (area) + spotCount + 1 (env)
    int maxDepth;
    int count;        // paths in the frame
    // material-sorted shading: extend appends each path to bucket 0 (miss) or its hit's BSDF type (1-5); shade
    // consumes the buckets in order, so that a warp runs one BSDF's code
    int* sortQueue;   // [kSortKeys * count] or null (sorting off)
    int* sortCount;   // [(maxDepth + 1) * kSortKeys]
    int tailPaths;    // a bounce queue shorter than this is finished by kTail (0: wavefront to the end)
    unsigned int* errorFlags;   // bit 0: traversal stack overflow; bit 1: malformed tree (index out of range)
    // ray reordering between bounces (raySortBits > 0): for bounces 1..raySortBounces with at least
    // kRaySortMinRays rays, shade records each surviving path's bin -- its direction octant, then its origin
    // cell (raySortBits bits per axis over the cube |x| <= sceneMaxAbs, Morton order) -- beside its queue entry
    // and counts the bins; kRayBins turns the counts into bin starts and kRayScatter writes the queue in bin
    // order, which extend walks, so a warp traces rays of one octant from one region.
    int* rayBin;      // [count] bin of next-bounce queue slot i
    int* binCount;    // [(raySortBounces + 1) << (3 + 3 * raySortBits)] counts per bounce, then bin positions
    int* sortedQueue; // [count] the bounce's queue in bin order
    int raySortBits;  // origin cell bits per axis, 0 (off) to 4
    int raySortBounces;
    // one launch sequence over several scenes' views (bte_render_scene_batch): the frame's scene table and the
    // scene of every path (its view's); null in single-scene frames
    const DevScene* scenes;   // [sceneCount]
    uint8_t* pathScene;       // [count]
    int sceneCount;
    // path-ordered queues for the first orderBounces bounces (material-sorted shading on, ray reordering off):
    // extend records each path's bucket in pathKey instead of appending it, shade records kKeyNext or kKeyDead,
    // and a stable compaction over path indices (kOrderCompact) writes the material buckets and the next
    // bounce's queue in ascending path order, so that the 32 paths of a warp are neighbours in the path-state
    // arrays (float4 entries share 32-byte sectors) instead of scattered
    uint8_t* pathKey;         // [count rounded up to kOrderTile]
    unsigned long long* orderStatus;   // [2 * orderBounces][tiles][kSortKeys] look-back words, zeroed per frame
    int* orderTicket;         // [2 * orderBounces] tile tickets, zeroed per frame
    int orderBounces;
};
constexpr int kRaySortMinRays = 32768;
constexpr int kOrderTile = 8192;            // paths per tile of the ordered compaction (256 threads x 32)
constexpr uint8_t kKeyNext = 6;             // pathKey: the path continues to the next bounce
constexpr uint8_t kKeyDead = 0xff;          // pathKey: the path has ended
static_assert(kKeyNext >= kSortKeys, "next-bounce key distinct from the material buckets");

// One camera view of a batched frame (bte_render_views): its paths are
// [pathOffset, pathOffset + width*height*spp) of the frame, sample-major as
// in a single-view frame, and its pixels [pixelOffset, + width*height) of
// the frame's pixel space.
struct ViewDesc {
    CameraData cam;
    float tanHalf;
    int width, height, spp;
    uint32_t frameIndex;          // samples of this view accumulated before this frame
    int pathOffset, pixelOffset;
    int scene;                    // entry of the frame's scene table (several scenes in one launch sequence)
    float* accum;                 // [W*H*3] FP32 running mean
    double* accumD;               // [W*H*3] FP64 running sum
    uint32_t* framebuffer;        // [W*H] packed RGBA8
};

struct FrameParams {
    int width, height, spp;
    const uint32_t* frameIndex;   // device word: samples accumulated before this frame (read by the kernels,
                                  // so a captured frame graph replays with a new value)
    int rrStart;
    float tanHalf;
    CameraData cam;
    const ViewDesc* views;        // batched views (viewCount > 0) instead of the single camera above
    int viewCount;
};

}  // namespace bte
