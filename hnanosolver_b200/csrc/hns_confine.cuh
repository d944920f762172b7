// Vorticity confinement (vorticityConfinement, src/Cuda/Kernel.cu:682-727, with the curl of
// computeVorticityMag, src/Cuda/Utils.cuh:226-243) on a leaf tile in shared memory.
//
// A voxel's force needs the curl at the voxel and |curl| at the voxels fs away along each axis
// (fs = int(factorScale)); each curl reads the six face neighbours. For |fs| <= 1 every value a
// leaf needs lies in the box of local coordinates [-2, 9]^3 around it: the tile stages that box's
// velocity once (0 outside the domain), computes the curl and its magnitude once for each cell of
// [-1, 8]^3, and each voxel then reads its curl and the six magnitudes from shared memory. The
// gather form recomputes the 7 curls of every voxel from 42 global vec3 reads; the values and the
// order of every operation are the same, so are the results.
#pragma once

#include <cuda_runtime.h>

#include "hns_stencil.cuh"
#include "hns_types.cuh"

namespace hns {
namespace dev {

constexpr int kConfVB = 12;               // velocity box edge: local -2 .. 9
constexpr int kConfWB = 10;               // curl box edge: local -1 .. 8
constexpr int kConfVCells = kConfVB * kConfVB * kConfVB;
constexpr int kConfWCells = kConfWB * kConfWB * kConfWB;

struct ConfineTile {
    float v[3][kConfVCells];  // velocity, 0 outside the domain
    float w[3][kConfWCells];  // curl * factor
    float m[kConfWCells];     // |curl * factor|
};

__device__ __forceinline__ int conf_vi(int a, int b, int d) { return ((a + 2) * kConfVB + (b + 2)) * kConfVB + (d + 2); }
__device__ __forceinline__ int conf_wi(int a, int b, int d) { return ((a + 1) * kConfWB + (b + 1)) * kConfWB + (d + 1); }
__device__ __forceinline__ int conf_nbr(int a) { return a < 0 ? 0 : (a > 7 ? 2 : 1); }

// Stages the velocity box and computes the curl box of the CTA's leaf (L staged). Ends with a
// barrier: the tile is then read-only.
template <typename V>
__device__ __forceinline__ void confine_tile(const LeafNbhd& L, const V* __restrict__ vel, ConfineTile& T, float factor) {
    for (int c = threadIdx.x; c < kConfVCells; c += blockDim.x) {
        const int a = c / (kConfVB * kConfVB) - 2, b = (c / kConfVB) % kConfVB - 2, d = c % kConfVB - 2;
        const int l = L.nb[conf_nbr(a) * 9 + conf_nbr(b) * 3 + conf_nbr(d)];
        float3 u = make_float3(0.f, 0.f, 0.f);
        if (l >= 0) u = vload(vel, ((int64_t)l << 9) + local_offset(a, b, d));
        T.v[0][c] = u.x, T.v[1][c] = u.y, T.v[2][c] = u.z;
    }
    __syncthreads();
    constexpr int X = kConfVB * kConfVB, Y = kConfVB;
    for (int c = threadIdx.x; c < kConfWCells; c += blockDim.x) {
        const int a = c / (kConfWB * kConfWB) - 1, b = (c / kConfWB) % kConfWB - 1, d = c % kConfWB - 1;
        const int q = conf_vi(a, b, d);
        // (py.z - my.z) - (pz.y - mz.y), (pz.x - mz.x) - (px.z - mx.z), (px.y - mx.y) - (py.x - my.x)
        const float ox = ((T.v[2][q + Y] - T.v[2][q - Y]) - (T.v[1][q + 1] - T.v[1][q - 1])) * factor;
        const float oy = ((T.v[0][q + 1] - T.v[0][q - 1]) - (T.v[2][q + X] - T.v[2][q - X])) * factor;
        const float oz = ((T.v[1][q + X] - T.v[1][q - X]) - (T.v[0][q + Y] - T.v[0][q - Y])) * factor;
        T.w[0][c] = ox, T.w[1][c] = oy, T.w[2][c] = oz;
        T.m[c] = __fsqrt_rn(ox * ox + oy * oy + oz * oz);
    }
    __syncthreads();
}

// The confinement force's velocity at local voxel (a, b, d) of the tile: u + scale (N x omega) dt.
__device__ __forceinline__ float3 confine_at(const ConfineTile& T, int a, int b, int d, int fs, float inv_dx, float dt,
                                             float scale) {
    const int c = conf_wi(a, b, d);
    const float ox = T.w[0][c], oy = T.w[1][c], oz = T.w[2][c];
    const float mpx = T.m[conf_wi(a + fs, b, d)], mmx = T.m[conf_wi(a - fs, b, d)];
    const float mpy = T.m[conf_wi(a, b + fs, d)], mmy = T.m[conf_wi(a, b - fs, d)];
    const float mpz = T.m[conf_wi(a, b, d + fs)], mmz = T.m[conf_wi(a, b, d - fs)];
    const float gx = (mpx - mmx) * 0.5f * inv_dx;
    const float gy = (mpy - mmy) * 0.5f * inv_dx;
    const float gz = (mpz - mmz) * 0.5f * inv_dx;
    const float glen = sqrtf(gx * gx + gy * gy + gz * gz) + 1e-5f;
    const float nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const int q = conf_vi(a, b, d);
    const float3 u = make_float3(T.v[0][q], T.v[1][q], T.v[2][q]);
    const float fx = scale * (ny * oz - nz * oy), fy = scale * (nz * ox - nx * oz), fz = scale * (nx * oy - ny * ox);
    return make_float3(u.x + fx * dt, u.y + fy * dt, u.z + fz * dt);
}

}  // namespace dev
}  // namespace hns
