/*
 * oracle/ref_shim/optix.h -- ORACLE (test infrastructure only).
 *
 * The OptiX SDK is not available, and the layout check of ref_layout.cpp only
 * needs the two things optix_launch_params.h takes from it: the traversable
 * handle type (OptiX defines it as an unsigned 64-bit integer) and the SBT
 * record constants used by its SbtRecord template (the documented values:
 * 16-byte record alignment, 32-byte header).
 */
#ifndef BTE_REF_SHIM_OPTIX_H
#define BTE_REF_SHIM_OPTIX_H
typedef unsigned long long OptixTraversableHandle;
#define OPTIX_SBT_RECORD_ALIGNMENT 16
#define OPTIX_SBT_RECORD_HEADER_SIZE 32
#ifndef __align__
#define __align__(n) alignas(n)
#endif
#endif
