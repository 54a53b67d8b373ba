/*
 * Host shim for compiling the reference's CUDA kernel sources (.cuh) as
 * plain C++ -- TEST INFRASTRUCTURE ONLY.  It maps the CUDA execution-space
 * qualifiers to nothing, the built-in thread/block indices to host globals
 * that a serial launch loop sets, __syncthreads() to a no-op, and supplies
 * the few int3/Float operators the reference takes from NVIDIA's
 * helper_math.h (which is not shipped with the reference).
 */
#ifndef REF_SHIM_H_
#define REF_SHIM_H_

#include <cmath>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>
#include <vector_functions.h>

#undef __global__
#undef __device__
#undef __host__
#undef __constant__
#undef __shared__
#undef __forceinline__
#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#define __forceinline__ inline

/* Built-in indices, set by the serial launch loop in ref_host.cpp. */
extern uint3 ref_threadIdx, ref_blockIdx;
extern dim3 ref_blockDim, ref_gridDim;
#define threadIdx ref_threadIdx
#define blockIdx ref_blockIdx
#define blockDim ref_blockDim
#define gridDim ref_gridDim

inline void __syncthreads() {}

/* helper_math.h-style operators used by the reference kernels */
inline int3 operator+(int3 a, int3 b) { return make_int3(a.x + b.x, a.y + b.y, a.z + b.z); }

#endif
