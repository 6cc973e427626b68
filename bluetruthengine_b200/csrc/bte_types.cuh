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

struct DevScene {
    // geometry
    const TriangleData* tris;         // reference AoS, original triangle order
    int triCount;
    const float4* leafTris;           // [triCount*3] v0.xyz|origIndex, v1.xyz, v2.xyz in leaf order
    const BvhNode* nodes;             // root = node 0 (triCount >= 2) or a single-leaf root
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
    int* shadowQueue; // entries path*slots + slot
    float4* shOrigin; // [paths] hit point of the NEE rays of the current bounce
    float4* shDir;    // [paths*slots] direction | tmax
    float4* shContrib;// [paths*slots] contribution | unused
    uint32_t* shMask; // [paths] bit s: slot s visible and not yet added
    int* hitLog;      // optional [paths*maxDepth]
    int slots;        // 1 (area) + spotCount + 1 (env)
    int maxDepth;
    int count;        // paths in the frame
    unsigned int* errorFlags;   // bit 0: traversal stack overflow
};

struct FrameParams {
    int width, height, spp;
    uint32_t frameIndex;          // samples accumulated before this frame
    int rrStart;
    float tanHalf;
    CameraData cam;
};

}  // namespace bte
