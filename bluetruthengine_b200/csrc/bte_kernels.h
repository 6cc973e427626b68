// bte_kernels.h -- host-side launchers of the device code (bte_kernels.cu,
// bte_bvh.cu, bte_env.cu).
#pragma once

#include "bte_types.cuh"

#include <string>

namespace bte {

void launchGenerate(const DevPaths& P, const FrameParams& f, cudaStream_t st);
void launchExtend(const DevScene& s, const DevPaths& P, int bounce, int grid, int block, cudaStream_t st);
// bounce's queue into ray-bin order before its extend (no-op unless DevPaths.raySortBits and the bounce qualify)
void launchRaySort(const DevPaths& P, int bounce, int grid, cudaStream_t st);
// ordered compaction of a path-ordered bounce: the material buckets (after extend) or the next queue (after shade)
int orderTiles(int paths);
void launchOrder(const DevPaths& P, int bounce, bool nextQueue, cudaStream_t st);
void launchShade(const DevScene& s, const DevPaths& P, const FrameParams& f, int bounce, int grid, int block,
                 int minBlocks, cudaStream_t st);
void launchConnect(const DevScene& s, const DevPaths& P, int bounce, int grid, int block, cudaStream_t st);
void launchTail(const DevScene& s, const DevPaths& P, const FrameParams& f, cudaStream_t st);
void launchMegakernel(const DevScene& s, const DevPaths& P, const FrameParams& f, float* accum, double* accumD,
                      uint32_t* fb, uint32_t* extFb, float* aovAccum, cudaStream_t st);
void launchPresentViews(const DevPaths& P, const FrameParams& f, int totalPixels, cudaStream_t st);
void launchPresent(const DevPaths& P, const FrameParams& f, float* accum, double* accumD, uint32_t* fb, uint32_t* extFb,
                   float* aovAccum, cudaStream_t st);
// lanes 1: one lane per ray (the tree in use); lanes 8: eight lanes per ray (8-wide tree only)
void launchTraceClosestRays(const DevScene& s, const float* rays, int n, int* outTri, float* outTuv, unsigned int* err,
                            int lanes, cudaStream_t st);
void launchTraceOccludedRays(const DevScene& s, const float* rays, const float* tmax, int n, uint8_t* out,
                             unsigned int* err, int lanes, cudaStream_t st);
void launchEnvQuery(const DevScene& s, int op, const float* in, int n, float* out, cudaStream_t st);
void launchMathEval(int fn, const float* a, const float* b, float* out, int n, cudaStream_t st);
void launchBsdfQuery(const BsdfData& g, int op, const float* wi, const float* x, int n, float* out, cudaStream_t st);
void launchTexCompare(cudaTextureObject_t tex, const float4* texels, int w, int h, int wrapV, const float* uv, int n,
                      float* outHw, float* outSw, cudaStream_t st);
int occupancyGrid(int which, int block);
void launchPackImage(const float* rgb, int n, uint32_t* fb, uint32_t* extFb, cudaStream_t st);

// LBVH build over device triangles (bte_bvh.cu).  Allocates `nodes` and
// `leafTris`; the caller frees them.  Returns 0 or a CUDA error code.
// width 2: BVH2 `nodes`; width 8: the 8-wide tree `wnodes` collapsed from the
// same binary tree.  `leafTris` is in the leaf order of the tree built.
struct BvhBuildResult {
    BvhNode* nodes = nullptr;
    WideNode* wnodes = nullptr;
    float4* leafTris = nullptr;
    int width = 2;
    int nodeCount = 0;
    int depth = 0;          // levels of the 8-wide tree
    int rootIsLeaf = 0;
    int rootCode = ~0;      // leaf code of the root when rootIsLeaf
    int builder = 0;        // hierarchy built: 0 Morton-prefix (Karras), 1 PLOC
    float msBuild = 0.0f;
};
// builder 1 asks for PLOC with neighbour search radius `radius`; a binary
// tree too deep for the traversal stack falls back to the Morton-prefix one.
// wideCollapse: 0 greedy (largest surface area opened first), 1 surface-area-optimal dynamic program
int buildLbvh(const TriangleData* dTris, int triCount, int maxLeaf, int width, int builder, int radius, int wideCollapse,
              BvhBuildResult& out, cudaStream_t st, std::string& err);

// The LBVH's Morton codes (per triangle, before sorting) and its stable sorted order, for host triangles.
int lbvhMortonOrder(const TriangleData* hostTris, int n, unsigned long long* hostKeys, int* hostSorted,
                    std::string& err);

// Env-map tables (bte_env.cu).
int buildEnvCdf(const float4* dTexels, int w, int h, const float* hSinTheta, float* dMarginal, float* dConditional,
                cudaStream_t st, std::string& err);
int buildEnvAlias(const float4* dTexels, int w, int h, float* dRowProb, int* dRowAlias, float* dColProb, int* dColAlias,
                  float* dPixelPdf, double* hTotal, cudaStream_t st, std::string& err);
// Device address lookup of bte_env_build_alias_noalloc's scratch array on the current device.
int prepareEnvNoallocScratch(std::string& err);

}  // namespace bte
