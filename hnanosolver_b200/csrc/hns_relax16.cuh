// The red-black update of the FP16 inner solve, shared by its kernels so that every layout gives
// the same values to the bit: FP16 operands, FP32 arithmetic, one FP16 rounding at the end.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "hns_stencil.cuh"

namespace hns {
namespace relax16 {

// FP16 operand (low 16 bits of h) into FP32 arithmetic: h + c, and a * b + c, rounded once.
__device__ __forceinline__ float addh(uint32_t h, float c) {
    float d;
    asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"((unsigned short)h), "f"(c));
    return d;
}
__device__ __forceinline__ float fmah(uint32_t a, uint32_t b, float c) {
    float d;
    asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"((unsigned short)a), "h"((unsigned short)b), "f"(c));
    return d;
}
__device__ __forceinline__ float h2f(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)h)); }

constexpr uint32_t kHalfMinusOne = 0xBC00u;

// One update of redBlackGaussSeidelUpdate with dx^2 = 1, as rbgs_stream_kernel<__half> does it:
// sum = x+ + x- + y+ + y- + z+ + z- (FP32, in that order), pgs = (sum - b) times the
// reference's 1/6, result = c + omega (pgs - c), rounded to FP16 by the caller. The FP16
// operands enter the FP32 operations directly (their conversion is exact).
__device__ __forceinline__ float relax1(uint32_t xp, uint32_t xm, uint32_t yp, uint32_t ym, uint32_t zp, uint32_t zm,
                                        uint32_t b, uint32_t c, float omega) {
    float s = h2f(xp);
    s = addh(xm, s);
    s = addh(yp, s);
    s = addh(ym, s);
    s = addh(zp, s);
    s = addh(zm, s);
    const float pgs = fmah(b, kHalfMinusOne, s) * dev::kInv6;  // (sum - b * 1) / 6
    const float d = fmah(c, kHalfMinusOne, pgs);              // pgs - c
    return addh(c, omega * d);                                 // c + omega (pgs - c)
}

// The same on the two halves of packed pairs; returns the packed FP16 results.
__device__ __forceinline__ uint32_t relax2(uint32_t xp, uint32_t xm, uint32_t yp, uint32_t ym, uint32_t zp, uint32_t zm,
                                           uint32_t b, uint32_t c, float omega) {
    const float lo = relax1(xp, xm, yp, ym, zp, zm, b, c, omega);
    const float hi = relax1(xp >> 16, xm >> 16, yp >> 16, ym >> 16, zp >> 16, zm >> 16, b >> 16, c >> 16, omega);
    const __half2 r = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&r);
}

__device__ __forceinline__ uint32_t round_half(float v) { return __half_as_ushort(__float2half_rn(v)); }

}  // namespace relax16
}  // namespace hns
