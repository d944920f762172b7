// Host-compilation shim for the reference's CUDA kernel source (src/Cuda/Kernel.cu).
//
// Test infrastructure only: it lets g++ compile the reference kernels unmodified as
// plain host functions, so that the oracle can run the reference's own arithmetic on
// the CPU. Each __global__ function becomes an ordinary function; the launch driver
// (ref_driver.cpp) sets the thread-local blockIdx/threadIdx/blockDim before each call.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime_api.h>  // declarations only (cudaMalloc, cudaEvent_t, ...): never called here

#undef __global__
#undef __device__
#undef __host__
#undef __forceinline__
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#ifndef __inline__
#define __inline__ inline
#endif

struct hns_shim_uint3 {
    unsigned int x, y, z;
};
extern thread_local hns_shim_uint3 blockIdx;
extern thread_local hns_shim_uint3 threadIdx;
extern thread_local hns_shim_uint3 blockDim;

// CUDA device intrinsics used by the reference, mapped to their IEEE host equivalents.
inline float __fmaf_rn(float a, float b, float c) { return std::fma(a, b, c); }
inline int __float2int_rd(float x) { return static_cast<int>(std::floor(x)); }
inline float __fsqrt_rn(float x) { return std::sqrt(x); }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fsub_rn(float a, float b) { return a - b; }
