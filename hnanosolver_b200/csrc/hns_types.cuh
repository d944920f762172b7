// Storage types of the solver's fields and their loads/stores as FP32.
//
// FP32 path: scalars float, vec3 float[3] interleaved.
// Mixed path: scalars FP16 (__half), vec3 BF16[3] interleaved (6 bytes per voxel).
// Arithmetic is FP32 in both; values are rounded to nearest when stored.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace hns {
namespace dev {

__device__ __forceinline__ float sload(const float* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ float sload(const __half* p, int64_t i) { return __half2float(__ldg(p + i)); }
__device__ __forceinline__ float sload(const double* p, int64_t i) { return (float)__ldg(p + i); }

__device__ __forceinline__ void sstore(float* p, int64_t i, float v) { p[i] = v; }
__device__ __forceinline__ void sstore(__half* p, int64_t i, float v) { p[i] = __float2half_rn(v); }

__device__ __forceinline__ float3 vload(const float* p, int64_t s) {
    return make_float3(__ldg(p + 3 * s), __ldg(p + 3 * s + 1), __ldg(p + 3 * s + 2));
}
__device__ __forceinline__ float3 vload(const __nv_bfloat16* p, int64_t s) {
    return make_float3(__bfloat162float(__ldg(p + 3 * s)), __bfloat162float(__ldg(p + 3 * s + 1)),
                       __bfloat162float(__ldg(p + 3 * s + 2)));
}

__device__ __forceinline__ void vstore(float* p, int64_t s, float3 v) {
    p[3 * s] = v.x;
    p[3 * s + 1] = v.y;
    p[3 * s + 2] = v.z;
}
__device__ __forceinline__ void vstore(__nv_bfloat16* p, int64_t s, float3 v) {
    p[3 * s] = __float2bfloat16_rn(v.x);
    p[3 * s + 1] = __float2bfloat16_rn(v.y);
    p[3 * s + 2] = __float2bfloat16_rn(v.z);
}

}  // namespace dev
}  // namespace hns
