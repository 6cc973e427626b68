/*
 * oracle/ref_shim/cuda_runtime.h -- ORACLE build shim (test infrastructure).
 *
 * Stands in for the CUDA runtime header so that the reference's trace-free
 * shading headers (include/rt_*.cuh, include/wavefront/*.cuh) compile as
 * plain host C++ with g++.  Execution-space qualifiers become inline, the
 * vector types are PODs, tex2D<> is routed to the oracle's emulation of the
 * documented linear-filtering formula, rsqrtf is 1/sqrtf (the same choice the
 * oracle and the GPU kernels make), and M_PI is pinned to the float literal
 * that rt_env_map.cuh:26-28 intends.
 */
#ifndef BTE_REF_SHIM_CUDA_RUNTIME_H
#define BTE_REF_SHIM_CUDA_RUNTIME_H

#include <cmath>
#include <cstdint>
#include <cstring>

#undef M_PI
#define M_PI 3.14159265358979323846f

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __constant__

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct uint3 { unsigned int x, y, z; };
struct uchar4 { unsigned char x, y, z, w; };

typedef unsigned long long cudaTextureObject_t;

inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline int atomicAdd(int* p, int v) { const int o = *p; *p = o + v; return o; }
inline float atomicAdd(float* p, float v) { const float o = *p; *p = o + v; return o; }

/* Texture registry owned by the harness: handle -> emulated texture. */
extern "C" float4 bte_ref_tex2d_float4(cudaTextureObject_t obj, float u, float v);
template <typename T> T tex2D(cudaTextureObject_t obj, float u, float v);
template <> inline float4 tex2D<float4>(cudaTextureObject_t obj, float u, float v)
{
    return bte_ref_tex2d_float4(obj, u, v);
}

#endif
