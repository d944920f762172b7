// Device-side helpers shared by the solver kernels: leaf lookup, slot addressing and the
// samplers of the reference (src/Utils/Stencils.hpp) restated over the leaf table.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "hns_internal.cuh"

namespace hns {
namespace dev {

constexpr float kInv6 = 0.166666667f;  // the reference's constant (src/Cuda/Kernel.cu:475)

__device__ __forceinline__ int local_offset(int i, int j, int k) { return ((i & 7) << 6) | ((j & 7) << 3) | (k & 7); }

// Leaf index of the voxel (i,j,k) through the dense leaf table, -1 outside the domain.
__device__ __forceinline__ int leaf_from_table(const TopoView& t, int i, int j, int k) {
    const int a = (i >> 3) - t.lo_x, b = (j >> 3) - t.lo_y, c = (k >> 3) - t.lo_z;
    if ((unsigned)a >= (unsigned)t.dim_x || (unsigned)b >= (unsigned)t.dim_y || (unsigned)c >= (unsigned)t.dim_z) return -1;
    return __ldg(t.lookup + ((int64_t)a * t.dim_y + b) * t.dim_z + c);
}

// The 27-leaf neighbourhood of the leaf a CTA works on, staged in shared memory.
struct LeafNbhd {
    int nb[27];
    int lx, ly, lz;  // leaf coordinates (origin >> 3)
};

__device__ __forceinline__ void load_nbhd(LeafNbhd& L, const TopoView& t, int64_t leaf) {
    if (threadIdx.x < 27) L.nb[threadIdx.x] = __ldg(t.nbr27 + leaf * 27 + threadIdx.x);
    if (threadIdx.x == 27) {
        const int4 o = t.origin[leaf];
        L.lx = o.x >> 3;
        L.ly = o.y >> 3;
        L.lz = o.z >> 3;
    }
}

__device__ __forceinline__ int leaf_of(const TopoView& t, const LeafNbhd& L, int i, int j, int k) {
    const int a = (i >> 3) - L.lx + 1, b = (j >> 3) - L.ly + 1, c = (k >> 3) - L.lz + 1;
    if ((unsigned)a < 3u && (unsigned)b < 3u && (unsigned)c < 3u) return L.nb[a * 9 + b * 3 + c];
    return leaf_from_table(t, i, j, k);
}

// Slot of voxel (i,j,k), -1 outside the domain.
__device__ __forceinline__ int64_t slot_of(const TopoView& t, const LeafNbhd& L, int i, int j, int k) {
    const int l = leaf_of(t, L, i, j, k);
    return l < 0 ? -1 : ((int64_t)l << 9) + local_offset(i, j, k);
}

__device__ __forceinline__ float3 ld3(const float* __restrict__ v, int64_t s) {
    return make_float3(__ldg(v + 3 * s), __ldg(v + 3 * s + 1), __ldg(v + 3 * s + 2));
}

__device__ __forceinline__ void st3(float* __restrict__ v, int64_t s, float3 a) {
    v[3 * s] = a.x;
    v[3 * s + 1] = a.y;
    v[3 * s + 2] = a.z;
}

// Nearest reads, 0 outside the domain (IndexSampler<T,0>, src/Utils/Stencils.hpp:74-93).
__device__ __forceinline__ float near_s(const TopoView& t, const LeafNbhd& L, const float* __restrict__ d, int i, int j, int k) {
    const int64_t s = slot_of(t, L, i, j, k);
    return s < 0 ? 0.f : __ldg(d + s);
}

__device__ __forceinline__ float3 near_v(const TopoView& t, const LeafNbhd& L, const float* __restrict__ d, int i, int j, int k) {
    const int64_t s = slot_of(t, L, i, j, k);
    return s < 0 ? make_float3(0.f, 0.f, 0.f) : ld3(d, s);
}

// a + w (b - a), rounded after each operation (the reference's sampler lerp,
// src/Utils/Stencils.hpp:137-140; the library is built without implicit FMA contraction).
__device__ __forceinline__ float lerp1(float a, float b, float w) { return a + w * (b - a); }

// Trilinear sample, 0 outside the domain: floor, fractional part, lerp along z, then y,
// then x (TrilinearSampler::sample, src/Utils/Stencils.hpp:118-153).
__device__ __forceinline__ float tri_s(const TopoView& t, const LeafNbhd& L, const float* __restrict__ d, float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
    const float v000 = near_s(t, L, d, i, j, k), v001 = near_s(t, L, d, i, j, k + 1);
    const float v010 = near_s(t, L, d, i, j + 1, k), v011 = near_s(t, L, d, i, j + 1, k + 1);
    const float v100 = near_s(t, L, d, i + 1, j, k), v101 = near_s(t, L, d, i + 1, j, k + 1);
    const float v110 = near_s(t, L, d, i + 1, j + 1, k), v111 = near_s(t, L, d, i + 1, j + 1, k + 1);
    const float z0 = lerp1(v000, v001, tz), z1 = lerp1(v010, v011, tz);
    const float z2 = lerp1(v100, v101, tz), z3 = lerp1(v110, v111, tz);
    return lerp1(lerp1(z0, z1, ty), lerp1(z2, z3, ty), tx);
}

__device__ __forceinline__ float3 tri_v(const TopoView& t, const LeafNbhd& L, const float* __restrict__ d, float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
    const float3 v000 = near_v(t, L, d, i, j, k), v001 = near_v(t, L, d, i, j, k + 1);
    const float3 v010 = near_v(t, L, d, i, j + 1, k), v011 = near_v(t, L, d, i, j + 1, k + 1);
    const float3 v100 = near_v(t, L, d, i + 1, j, k), v101 = near_v(t, L, d, i + 1, j, k + 1);
    const float3 v110 = near_v(t, L, d, i + 1, j + 1, k), v111 = near_v(t, L, d, i + 1, j + 1, k + 1);
    float3 r;
#define HNS_TRI_COMP(c)                                                                   \
    {                                                                                     \
        const float z0 = lerp1(v000.c, v001.c, tz), z1 = lerp1(v010.c, v011.c, tz);       \
        const float z2 = lerp1(v100.c, v101.c, tz), z3 = lerp1(v110.c, v111.c, tz);       \
        r.c = lerp1(lerp1(z0, z1, ty), lerp1(z2, z3, ty), tx);                            \
    }
    HNS_TRI_COMP(x)
    HNS_TRI_COMP(y)
    HNS_TRI_COMP(z)
#undef HNS_TRI_COMP
    return r;
}

// The eight taps of a trilinear sample at (x,y,z): slots (-1 outside the domain) of the
// corners v[a][b][c] = (i+a, j+b, k+c) and the fractional position. Computing them once
// lets several fields be sampled at the same point with shared addressing.
// I: the slot type, int64_t in general, int32_t where the grid has fewer than 2^22 leaves
// (32-bit address arithmetic, half the integer instructions per tap).
template <typename I>
struct TapsT {
    I s[8];  // index a*4 + b*2 + c
    float tx, ty, tz;
};
using Taps = TapsT<int64_t>;

// The cell's two planes along each axis are resolved once: when both lie in the CTA leaf's
// 3x3x3 neighbourhood (every trace shorter than a leaf), each corner's leaf is one
// shared-memory lookup at a precomputed index and its slot an OR of precomputed local
// offsets; otherwise every corner goes through slot_of (and the leaf table).
template <typename I>
__device__ __forceinline__ void taps_at(TapsT<I>& T, const TopoView& t, const LeafNbhd& L, float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    T.tx = x - (float)i;
    T.ty = y - (float)j;
    T.tz = z - (float)k;
    const int a0 = (i >> 3) - L.lx + 1, a1 = ((i + 1) >> 3) - L.lx + 1;
    const int b0 = (j >> 3) - L.ly + 1, b1 = ((j + 1) >> 3) - L.ly + 1;
    const int c0 = (k >> 3) - L.lz + 1, c1 = ((k + 1) >> 3) - L.lz + 1;
    if ((unsigned)a0 < 3u && (unsigned)a1 < 3u && (unsigned)b0 < 3u && (unsigned)b1 < 3u && (unsigned)c0 < 3u &&
        (unsigned)c1 < 3u) {
        const int na[2] = {a0 * 9, a1 * 9}, nb[2] = {b0 * 3, b1 * 3}, nc[2] = {c0, c1};
        const int la[2] = {(i & 7) << 6, ((i + 1) & 7) << 6}, lb[2] = {(j & 7) << 3, ((j + 1) & 7) << 3};
        const int lc[2] = {k & 7, (k + 1) & 7};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int A = q >> 2, B = (q >> 1) & 1, C = q & 1;
            const int l = L.nb[na[A] + nb[B] + nc[C]];
            T.s[q] = l < 0 ? I(-1) : (I(l) << 9) + I(la[A] | lb[B] | lc[C]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) T.s[q] = (I)slot_of(t, L, i + (q >> 2), j + ((q >> 1) & 1), k + (q & 1));
    }
}

// Slots of the six face neighbours of local voxel n of the CTA's leaf (slot s), -1 outside the
// domain, in the order x-1, x+1, y-1, y+1, z-1, z+1: the leaf's own slots unless the
// neighbour is across a face, then the face neighbour from the staged neighbourhood.
template <typename I>
__device__ __forceinline__ void face_slots(const LeafNbhd& L, I s, int n, I ns[6]) {
    const int a = n >> 6, b = (n >> 3) & 7, c = n & 7;
    auto across = [&](int idx, int local) -> I {
        const int l = L.nb[idx];
        return l < 0 ? I(-1) : (I(l) << 9) + I(local);
    };
    ns[0] = a > 0 ? s - 64 : across(4, n | (7 << 6));
    ns[1] = a < 7 ? s + 64 : across(22, n & 63);
    ns[2] = b > 0 ? s - 8 : across(10, n | (7 << 3));
    ns[3] = b < 7 ? s + 8 : across(16, n & ~(7 << 3));
    ns[4] = c > 0 ? s - 1 : across(12, n | 7);
    ns[5] = c < 7 ? s + 1 : across(14, n & ~7);
}

__device__ __forceinline__ float tap_s(const float* __restrict__ d, int64_t s) { return s < 0 ? 0.f : __ldg(d + s); }

__device__ __forceinline__ float3 tap_v(const float* __restrict__ d, int64_t s) {
    return s < 0 ? make_float3(0.f, 0.f, 0.f) : ld3(d, s);
}

// Lerp along z, then y, then x of the staged corners (TrilinearSampler::sample order).
template <typename I>
__device__ __forceinline__ float tri_lerp(const TapsT<I>& T, const float v[8]) {
    const float z0 = lerp1(v[0], v[1], T.tz), z1 = lerp1(v[2], v[3], T.tz);
    const float z2 = lerp1(v[4], v[5], T.tz), z3 = lerp1(v[6], v[7], T.tz);
    return lerp1(lerp1(z0, z1, T.ty), lerp1(z2, z3, T.ty), T.tx);
}

__device__ __forceinline__ float tri_s(const Taps& T, const float* __restrict__ d) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = tap_s(d, T.s[q]);
    return tri_lerp(T, v);
}

__device__ __forceinline__ float3 tri_v(const Taps& T, const float* __restrict__ d) {
    float x[8], y[8], z[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float3 a = tap_v(d, T.s[q]);
        x[q] = a.x, y[q] = a.y, z[q] = a.z;
    }
    return make_float3(tri_lerp(T, x), tri_lerp(T, y), tri_lerp(T, z));
}

// Slot for the multi-field advection's taps: out-of-domain reads slot 0
// (src/Cuda/Kernel.cu:229-230, 256-257).
__device__ __forceinline__ int64_t tap_slot(const TopoView& t, const LeafNbhd& L, int i, int j, int k) {
    const int64_t s = slot_of(t, L, i, j, k);
    return s < 0 ? 0 : s;
}

// Eight taps and weights of the multi-field advection's weight-sum trilinear
// (setupInterpolation, src/Cuda/Kernel.cu:204-233).
__device__ __forceinline__ void interp_setup(const TopoView& t, const LeafNbhd& L, float x, float y, float z, int64_t idx[8], float w[8]) {
    const int i0 = __float2int_rd(x), j0 = __float2int_rd(y), k0 = __float2int_rd(z);
    const int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    const float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
    const float itx = 1.0f - tx, ity = 1.0f - ty, itz = 1.0f - tz;
    const float w00 = itx * ity, w10 = tx * ity, w01 = itx * ty, w11 = tx * ty;
    w[0] = w00 * itz;
    w[1] = w10 * itz;
    w[2] = w01 * itz;
    w[3] = w11 * itz;
    w[4] = w00 * tz;
    w[5] = w10 * tz;
    w[6] = w01 * tz;
    w[7] = w11 * tz;
    idx[0] = tap_slot(t, L, i0, j0, k0);
    idx[1] = tap_slot(t, L, i1, j0, k0);
    idx[2] = tap_slot(t, L, i0, j1, k0);
    idx[3] = tap_slot(t, L, i1, j1, k0);
    idx[4] = tap_slot(t, L, i0, j0, k1);
    idx[5] = tap_slot(t, L, i1, j0, k1);
    idx[6] = tap_slot(t, L, i0, j1, k1);
    idx[7] = tap_slot(t, L, i1, j1, k1);
}

// interp_setup with the taps' slots in I (int32_t where the grid has fewer than 2^22 leaves):
// the same weights and the same slots, the cell's planes resolved once as in taps_at when both
// lie in the CTA leaf's neighbourhood.
template <typename I>
__device__ __forceinline__ void interp_setup_fast(const TopoView& t, const LeafNbhd& L, float x, float y, float z,
                                                  I idx[8], float w[8]) {
    const int i0 = __float2int_rd(x), j0 = __float2int_rd(y), k0 = __float2int_rd(z);
    const int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    const float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
    const float itx = 1.0f - tx, ity = 1.0f - ty, itz = 1.0f - tz;
    const float w00 = itx * ity, w10 = tx * ity, w01 = itx * ty, w11 = tx * ty;
    w[0] = w00 * itz;
    w[1] = w10 * itz;
    w[2] = w01 * itz;
    w[3] = w11 * itz;
    w[4] = w00 * tz;
    w[5] = w10 * tz;
    w[6] = w01 * tz;
    w[7] = w11 * tz;
    const int a0 = (i0 >> 3) - L.lx + 1, a1 = (i1 >> 3) - L.lx + 1;
    const int b0 = (j0 >> 3) - L.ly + 1, b1 = (j1 >> 3) - L.ly + 1;
    const int c0 = (k0 >> 3) - L.lz + 1, c1 = (k1 >> 3) - L.lz + 1;
    if ((unsigned)a0 < 3u && (unsigned)a1 < 3u && (unsigned)b0 < 3u && (unsigned)b1 < 3u && (unsigned)c0 < 3u &&
        (unsigned)c1 < 3u) {
        const int na[2] = {a0 * 9, a1 * 9}, nb[2] = {b0 * 3, b1 * 3}, nc[2] = {c0, c1};
        const int la[2] = {(i0 & 7) << 6, (i1 & 7) << 6}, lb[2] = {(j0 & 7) << 3, (j1 & 7) << 3};
        const int lc[2] = {k0 & 7, k1 & 7};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int A = q & 1, B = (q >> 1) & 1, C = q >> 2;  // interp_setup's order: x fastest
            const int l = L.nb[na[A] + nb[B] + nc[C]];
            idx[q] = l < 0 ? I(0) : (I(l) << 9) + I(la[A] | lb[B] | lc[C]);  // outside: slot 0
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) idx[q] = (I)tap_slot(t, L, (q & 1) ? i1 : i0, (q & 2) ? j1 : j0, (q & 4) ? k1 : k0);
    }
}

// |curl u| at a voxel (computeVorticityMag, src/Cuda/Utils.cuh:226-243).
__device__ __forceinline__ float vort_mag(const TopoView& t, const LeafNbhd& L, const float* __restrict__ v, int i, int j, int k, float factor) {
    const float3 px = near_v(t, L, v, i + 1, j, k), mx = near_v(t, L, v, i - 1, j, k);
    const float3 py = near_v(t, L, v, i, j + 1, k), my = near_v(t, L, v, i, j - 1, k);
    const float3 pz = near_v(t, L, v, i, j, k + 1), mz = near_v(t, L, v, i, j, k - 1);
    const float ox = ((py.z - my.z) - (pz.y - mz.y)) * factor;
    const float oy = ((pz.x - mz.x) - (px.z - mx.z)) * factor;
    const float oz = ((px.y - mx.y) - (py.x - my.x)) * factor;
    return __fsqrt_rn(ox * ox + oy * oy + oz * oz);
}

// ---- collision (src/Cuda/Kernel.cu:81-158) ----

// isInCollision: the trilinear SDF sample (0 outside the domain) below 0.
__device__ __forceinline__ bool sdf_inside(const TopoView& t, const LeafNbhd& L, const float* __restrict__ sdf, float x,
                                           float y, float z) {
    return tri_s(t, L, sdf, x, y, z) < 0.f;
}

// The collision treatment of a velocity at voxel (i, j, k), slot s: 0 inside the collider
// (sdf < 0); within the 0.1 margin, the normal component blended out with weight
// 1 - sdf / ramp (applyNoSlipBoundary; ramp 0.1 in enforceCollisionBoundaries and
// subtractPressureGradient, 1.5 in advect_vector). The normal is getSDFNormal: central
// differences of the SDF times 0.5 inv_dx, scaled by 1 / length (NanoVDB's Vec3f / s) when
// the length exceeds 1e-6.
__device__ __forceinline__ void collide(const TopoView& t, const LeafNbhd& L, const float* __restrict__ sdf, int64_t s, int i,
                                        int j, int k, float inv_dx, float ramp, float3& v) {
    const float d = __ldg(sdf + s);
    if (d < 0.f) {
        v = make_float3(0.f, 0.f, 0.f);
    } else if (d < 0.1f) {
        const float h = 0.5f * inv_dx;
        const float gx = h * (near_s(t, L, sdf, i + 1, j, k) - near_s(t, L, sdf, i - 1, j, k));
        const float gy = h * (near_s(t, L, sdf, i, j + 1, k) - near_s(t, L, sdf, i, j - 1, k));
        const float gz = h * (near_s(t, L, sdf, i, j, k + 1) - near_s(t, L, sdf, i, j, k - 1));
        const float len = __fsqrt_rn(gx * gx + gy * gy + gz * gz);
        const float r = len > 1e-6f ? __frcp_rn(len) : 0.f;
        const float nx = r * gx, ny = r * gy, nz = r * gz;
        const float vdotn = v.x * nx + v.y * ny + v.z * nz;
        const float tx = v.x - vdotn * nx, ty = v.y - vdotn * ny, tz = v.z - vdotn * nz;
        const float blend = 1.f - __fdiv_rn(d, ramp);
        const float keep = 1.f - blend;
        v = make_float3(keep * v.x + blend * tx, keep * v.y + blend * ty, keep * v.z + blend * tz);
    }
}

// Voxel handled by this thread in the "two CTAs per leaf" kernels.
struct VoxelIdx {
    int64_t leaf;
    int n;  // local slot 0..511
};

__device__ __forceinline__ VoxelIdx voxel_of_block() {
    VoxelIdx v;
    v.leaf = (int64_t)(blockIdx.x >> 1);
    v.n = (int)(((blockIdx.x & 1u) << 8) | threadIdx.x);
    return v;
}

}  // namespace dev
}  // namespace hns
