// Mixed-precision step: fields stored in BF16 (velocity) and FP16 (scalars), arithmetic in
// FP32, and the pressure solve wrapped in iterative refinement whose outer residuals and
// accumulated pressure are FP64.
//
// Refinement (b = div dx^2, L p = sum of the 6 neighbours - 6 p, p = 0 outside the domain):
//   p = 0; r = b
//   repeat: s = rms(r); r^ = r / s in FP16; solve L e = r^ approximately with `inner`
//           red-black SOR iterations on FP16 storage from e = 0; p += s e (FP64);
//           r = b - L p (FP64, stored FP32), ||r||^2 (FP64)
//   until ||r|| <= tol ||b||.
// The inner iterations move 6 bytes per voxel instead of the FP32 solve's 12, and the outer
// FP64 residual removes the FP32 rounding floor of a plain FP32 solve. Every kernel of the
// loop reads the latest residual check on the device and returns at once when the
// tolerance is met, so the host enqueues the whole loop without synchronizing.
//
// The same refinement with FP32 inner storage (hns_step_plain with HNS_SOLVE_REFINE) is the
// FP32 form it is compared with.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "hns_internal.cuh"
#include "hns_stencil.cuh"
#include "hns_types.cuh"

namespace hns {
namespace {

using namespace dev;

constexpr int kThreads = 256;

unsigned leaf_blocks(const Context& c) { return (unsigned)(c.topo.num_leaves * 2); }

__device__ __forceinline__ bool converged(const double* check, double tol2) {
    return check != nullptr && check[0] <= tol2 * check[1];
}

// Block-wide FP64 sum of two values into acc[0], acc[1] (kBlock threads).
template <int kBlock = kThreads>
__device__ __forceinline__ void block_sum2(double a, double b, double* acc) {
    __shared__ double red[2][kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = a, red[1][threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        a = threadIdx.x < kBlock / 32 ? red[0][threadIdx.x] : 0.0;
        b = threadIdx.x < kBlock / 32 ? red[1][threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (threadIdx.x == 0) {
            atomicAdd(acc, a);
            atomicAdd(acc + 1, b);
        }
    }
}

// ---- advection on reduced-precision storage ---------------------------------------------

// Reduced-precision loads at a 32- or 64-bit slot (-1: outside the domain, read as 0). A 32-bit
// slot is widened in the multiply (one IMAD.WIDE per address).
__device__ __forceinline__ int64_t wide(int32_t s) { return (int64_t)(uint32_t)s; }
__device__ __forceinline__ int64_t wide(int64_t s) { return s; }

template <typename V, typename I>
__device__ __forceinline__ float3 tap3(const V* d, I s) {
    return s < 0 ? make_float3(0.f, 0.f, 0.f) : vload(d, wide(s));
}
template <typename S, typename I>
__device__ __forceinline__ float tap1(const S* d, I s) {
    return s < 0 ? 0.f : sload(d, wide(s));
}

template <typename V, typename I>
__device__ __forceinline__ float3 tri3(const TapsT<I>& T, const V* d) {
    float x[8], y[8], z[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float3 a = tap3(d, T.s[q]);
        x[q] = a.x, y[q] = a.y, z[q] = a.z;
    }
    return make_float3(tri_lerp(T, x), tri_lerp(T, y), tri_lerp(T, z));
}

template <typename S, typename I>
__device__ __forceinline__ float tri1(const TapsT<I>& T, const S* d) {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = tap1(d, T.s[q]);
    return tri_lerp(T, v);
}

template <typename S>
struct FieldSetT {
    const S* in[kMaxAdvectFields];
    S* out[kMaxAdvectFields];
    int count;
};

// advect_vector + advect_scalar along one shared trace (as advect_fused_kernel), reading and
// writing reduced-precision storage.
// I: the slot type (int32_t for fewer than 2^22 leaves). Four CTAs per SM (64 registers, no
// spills): 0.85 ms on a 45,198-leaf grid against 0.98 at three (80 registers).
template <typename V, typename S, typename I>
__global__ void __launch_bounds__(kThreads, 4) advect_mixed_kernel(TopoView t, const V* __restrict__ vel,
                                                                 V* __restrict__ vel_out, FieldSetT<S> f, float sdt) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const I s = (I(v.leaf) << 9) + I(v.n);
    const float3 vo = vload(vel, wide(s));
    const float bx = (float)i - vo.x * sdt, by = (float)j - vo.y * sdt, bz = (float)k - vo.z * sdt;
    TapsT<I> tb, tf;
    taps_at(tb, t, L, bx, by, bz);
    const float3 vf = tri3(tb, vel);
    taps_at(tf, t, L, bx + vf.x * sdt, by + vf.y * sdt, bz + vf.z * sdt);
    I ns[6];
    face_slots(L, s, v.n, ns);
    if (vel_out != nullptr) {
        const float3 vb = tri3(tf, vel);
        float3 corr = make_float3(vf.x + 0.5f * (vo.x - vb.x), vf.y + 0.5f * (vo.y - vb.y), vf.z + 0.5f * (vo.z - vb.z));
        float3 mn = vo, mx = vo;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float3 a = tap3(vel, ns[q]);
            mn.x = fminf(mn.x, a.x), mn.y = fminf(mn.y, a.y), mn.z = fminf(mn.z, a.z);
            mx.x = fmaxf(mx.x, a.x), mx.y = fmaxf(mx.y, a.y), mx.z = fmaxf(mx.z, a.z);
        }
        mn.x = fminf(mn.x, vf.x), mn.y = fminf(mn.y, vf.y), mn.z = fminf(mn.z, vf.z);
        mx.x = fmaxf(mx.x, vf.x), mx.y = fmaxf(mx.y, vf.y), mx.z = fmaxf(mx.z, vf.z);
        corr.x = fmaxf(mn.x, fminf(corr.x, mx.x));
        corr.y = fmaxf(mn.y, fminf(corr.y, mx.y));
        corr.z = fmaxf(mn.z, fminf(corr.z, mx.z));
        vstore(vel_out, wide(s), corr);
    }
    for (int c = 0; c < f.count; ++c) {
        const S* __restrict__ d = f.in[c];
        const float po = sload(d, wide(s));
        const float pf = tri1(tb, d);
        const float pb = tri1(tf, d);
        const float corr = pf + 0.5f * (po - pb);
        float mn = po, mx = po;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float a = tap1(d, ns[q]);
            mn = fminf(mn, a);
            mx = fmaxf(mx, a);
        }
        mn = fminf(mn, pf);
        mx = fmaxf(mx, pf);
        sstore(f.out[c], wide(s), fmaxf(mn, fminf(corr, mx)));
    }
}

// ---- stencils over half z-rows ------------------------------------------------------------
//
// The divergence, the gradient subtraction and the refinement residual are 7-point stencils in
// leaf slot order, where a leaf's z-row (x, y) = (a, b) is 8 contiguous slots. A thread covers
// z = 4h .. 4h + 3 of one row (128 threads per leaf, kRowLeaves leaves per 256-thread CTA): it
// loads its half row and the same half of the four x/y neighbour rows (the row of the leaf
// across a face at the leaf's edge; a missing leaf reads 0) as vector loads, and the two z
// neighbours past its ends (the row's other half, or the leaf across the z face). The leaves'
// face neighbours come straight from the 27-neighbour table: no staging, no barrier. Measured
// on a 45,198-leaf grid, one leaf per thread in 256-thread CTAs beat 128- and 512-thread CTAs
// and two or three leaves per thread for all three stencils.
constexpr int kRowLeaves = kThreads / 128;

struct HalfRow {
    int64_t leaf, own;   // own: slot of the half row's first voxel (a multiple of 4)
    int row, h, a, b;    // row = 8 a + b
    int nx, ny, nz;      // leaf across the x face / y face this row touches (itself inside), across
                         // the z face this half touches (-z for h = 0, +z for h = 1); -1 missing
};

// The half row of this thread in leaf group g (the kRowLeaves leaves one CTA covers); false
// past the last leaf.
__device__ __forceinline__ bool half_row(const TopoView& t, HalfRow& r, int64_t g) {
    r.leaf = g * kRowLeaves + (threadIdx.x >> 7);
    if (r.leaf >= t.num_leaves) return false;
    r.row = (threadIdx.x >> 1) & 63, r.h = threadIdx.x & 1, r.a = r.row >> 3, r.b = r.row & 7;
    r.own = (r.leaf << 9) + 8 * r.row + 4 * r.h;
    const int* nb = t.nbr27 + r.leaf * 27;
    // nbr27: (dx+1)*9 + (dy+1)*3 + (dz+1); entry 13 is the leaf itself.
    r.nx = __ldg(nb + (r.a == 7 ? 22 : r.a == 0 ? 4 : 13));
    r.ny = __ldg(nb + (r.b == 7 ? 16 : r.b == 0 ? 10 : 13));
    r.nz = __ldg(nb + (r.h ? 14 : 12));
    return true;
}

// Slots of the same half row in the four x/y neighbour rows (the half row itself where the
// neighbour leaf is missing: its values are then replaced by 0).
struct NbrRows {
    int64_t xp, xm, yp, ym;
    bool zxp, zxm, zyp, zym;  // missing neighbour: read as 0
};

__device__ __forceinline__ NbrRows nbr_rows(const HalfRow& r) {
    auto across = [&](int n, int rw) -> int64_t { return n < 0 ? r.own : ((int64_t)n << 9) + 8 * rw + 4 * r.h; };
    NbrRows q;
    q.xp = r.a < 7 ? r.own + 64 : across(r.nx, r.b);
    q.xm = r.a > 0 ? r.own - 64 : across(r.nx, 56 + r.b);
    q.yp = r.b < 7 ? r.own + 8 : across(r.ny, 8 * r.a);
    q.ym = r.b > 0 ? r.own - 8 : across(r.ny, 8 * r.a + 7);
    q.zxp = r.a == 7 && r.nx < 0, q.zxm = r.a == 0 && r.nx < 0, q.zyp = r.b == 7 && r.ny < 0, q.zym = r.b == 0 && r.ny < 0;
    return q;
}

// Slots of the z neighbours past the half row's ends: the row's other half, and the voxel
// across the z face (-1 when that leaf is missing).
__device__ __forceinline__ void z_ends(const HalfRow& r, int64_t& zin, int64_t& zface) {
    zin = r.h ? r.own - 1 : r.own + 4;
    zface = r.nz < 0 ? -1 : ((int64_t)r.nz << 9) + 8 * r.row + (r.h ? 0 : 7);
}

__device__ __forceinline__ void ld_half4(const double* __restrict__ q, double v[4]) {
    const double2 x0 = __ldg(reinterpret_cast<const double2*>(q));
    const double2 x1 = __ldg(reinterpret_cast<const double2*>(q) + 1);
    v[0] = x0.x, v[1] = x0.y, v[2] = x1.x, v[3] = x1.y;
}

// Velocity of four voxels from slot s (a multiple of 4): 12 interleaved components, 24 bytes in
// BF16 (three 8-byte loads) or 48 in FP32 (three 16-byte loads).
__device__ __forceinline__ float bf16_bits(uint32_t w, int hi) { return __uint_as_float(hi ? (w & 0xFFFF0000u) : (w << 16)); }

__device__ __forceinline__ void vel_half_row(const __nv_bfloat16* __restrict__ v, int64_t s, float3 u[4]) {
    const uint2* q = reinterpret_cast<const uint2*>(v + 3 * s);
    const uint2 w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
    const uint32_t w[6] = {w0.x, w0.y, w1.x, w1.y, w2.x, w2.y};
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        const int e = 3 * z;
        u[z] = make_float3(bf16_bits(w[e >> 1], e & 1), bf16_bits(w[(e + 1) >> 1], (e + 1) & 1),
                           bf16_bits(w[(e + 2) >> 1], (e + 2) & 1));
    }
}
__device__ __forceinline__ void vel_half_row(const float* __restrict__ v, int64_t s, float3 u[4]) {
    const float4* q = reinterpret_cast<const float4*>(v + 3 * s);
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    u[0] = make_float3(a.x, a.y, a.z);
    u[1] = make_float3(a.w, b.x, b.y);
    u[2] = make_float3(b.z, b.w, c.x);
    u[3] = make_float3(c.y, c.z, c.w);
}

__device__ __forceinline__ uint32_t bf16x2_bits(float lo, float hi) {
    const __nv_bfloat162 r = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&r);
}
__device__ __forceinline__ void store_vel_half_row(__nv_bfloat16* v, int64_t s, const float3 u[4]) {
    uint2* q = reinterpret_cast<uint2*>(v + 3 * s);
    q[0] = make_uint2(bf16x2_bits(u[0].x, u[0].y), bf16x2_bits(u[0].z, u[1].x));
    q[1] = make_uint2(bf16x2_bits(u[1].y, u[1].z), bf16x2_bits(u[2].x, u[2].y));
    q[2] = make_uint2(bf16x2_bits(u[2].z, u[3].x), bf16x2_bits(u[3].y, u[3].z));
}
__device__ __forceinline__ void store_vel_half_row(float* v, int64_t s, const float3 u[4]) {
    float4* q = reinterpret_cast<float4*>(v + 3 * s);
    q[0] = make_float4(u[0].x, u[0].y, u[0].z, u[1].x);
    q[1] = make_float4(u[1].y, u[1].z, u[2].x, u[2].y);
    q[2] = make_float4(u[2].z, u[3].x, u[3].y, u[3].z);
}

// Element-wise forms of the same, for velocity arrays that are not 8-byte (BF16) or 16-byte
// (FP32) aligned; kVec selects the vector form.
template <bool kVec, typename V>
__device__ __forceinline__ void vel_row(const V* __restrict__ v, int64_t s, float3 u[4]) {
    if constexpr (kVec) {
        vel_half_row(v, s, u);
    } else {
#pragma unroll
        for (int z = 0; z < 4; ++z) u[z] = vload(v, s + z);
    }
}
template <bool kVec, typename V>
__device__ __forceinline__ void store_vel_row(V* v, int64_t s, const float3 u[4]) {
    if constexpr (kVec) {
        store_vel_half_row(v, s, u);
    } else {
#pragma unroll
        for (int z = 0; z < 4; ++z) vstore(v, s + z, u[z]);
    }
}

__device__ __forceinline__ float vel_z(const __nv_bfloat16* __restrict__ v, int64_t s) {
    return __bfloat162float(__ldg(v + 3 * s + 2));
}

// Divergence (divergence, src/Cuda/Kernel.cu:432-453) of a reduced-precision velocity into
// FP32: per voxel the face velocities are the means of the centre and the neighbour (0 for a
// missing neighbour), div = (xp - xm + yp - ym + zp - zm) / dx.
template <typename V, bool kVec>
__global__ void __launch_bounds__(kThreads) divergence_mixed_kernel(TopoView t, const V* __restrict__ vel,
                                                                     float* __restrict__ div, float inv_dx) {
    HalfRow r;
    if (!half_row(t, r, blockIdx.x)) return;
    const NbrRows q = nbr_rows(r);
    float3 c[4], xp[4], xm[4], yp[4], ym[4];
    vel_row<kVec>(vel, r.own, c);
    vel_row<kVec>(vel, q.xp, xp);
    vel_row<kVec>(vel, q.xm, xm);
    vel_row<kVec>(vel, q.yp, yp);
    vel_row<kVec>(vel, q.ym, ym);
    int64_t zin_s, zface_s;
    z_ends(r, zin_s, zface_s);
    const float zin = vel_z(vel, zin_s), zface = zface_s < 0 ? 0.f : vel_z(vel, zface_s);
    const float zlo = r.h ? zin : zface, zhi = r.h ? zface : zin;
    float d[4];
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        const float vxp = (c[z].x + (q.zxp ? 0.f : xp[z].x)) * 0.5f;
        const float vxm = (c[z].x + (q.zxm ? 0.f : xm[z].x)) * 0.5f;
        const float vyp = (c[z].y + (q.zyp ? 0.f : yp[z].y)) * 0.5f;
        const float vym = (c[z].y + (q.zym ? 0.f : ym[z].y)) * 0.5f;
        const float vzp = (c[z].z + (z < 3 ? c[z + 1].z : zhi)) * 0.5f;
        const float vzm = (c[z].z + (z > 0 ? c[z - 1].z : zlo)) * 0.5f;
        d[z] = (vxp - vxm + vyp - vym + vzp - vzm) * inv_dx;
    }
    *reinterpret_cast<float4*>(div + r.own) = make_float4(d[0], d[1], d[2], d[3]);
}

// u -= grad p with p in FP64 (0 outside the domain), central differences
// (subtractPressureGradient, src/Cuda/Kernel.cu:495-541), velocity in reduced precision or
// FP32, in place.
template <typename V, bool kVec>
__global__ void __launch_bounds__(kThreads) gradient_mixed_kernel(TopoView t, V* __restrict__ vel,
                                                                   const double* __restrict__ p, float inv_dx) {
    HalfRow r;
    if (!half_row(t, r, blockIdx.x)) return;
    const NbrRows q = nbr_rows(r);
    double c[4], xp[4], xm[4], yp[4], ym[4];
    ld_half4(p + r.own, c);
    ld_half4(p + q.xp, xp);
    ld_half4(p + q.xm, xm);
    ld_half4(p + q.yp, yp);
    ld_half4(p + q.ym, ym);
    int64_t zin_s, zface_s;
    z_ends(r, zin_s, zface_s);
    const double zin = __ldg(p + zin_s), zface = zface_s < 0 ? 0.0 : __ldg(p + zface_s);
    const double zlo = r.h ? zin : zface, zhi = r.h ? zface : zin;
    float3 u[4];
    vel_row<kVec>(vel, r.own, u);
    const double hh = 0.5 * (double)inv_dx;
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        const float gx = (float)(((q.zxp ? 0.0 : xp[z]) - (q.zxm ? 0.0 : xm[z])) * hh);
        const float gy = (float)(((q.zyp ? 0.0 : yp[z]) - (q.zym ? 0.0 : ym[z])) * hh);
        const float gz = (float)(((z < 3 ? c[z + 1] : zhi) - (z > 0 ? c[z - 1] : zlo)) * hh);
        u[z] = make_float3(u[z].x - gx, u[z].y - gy, u[z].z - gz);
    }
    store_vel_row<kVec>(vel, r.own, u);
}

// ---- refinement --------------------------------------------------------------------------

// r = b - L p (FP64 arithmetic, r stored FP32) with b = div dx^2 and p = 0 outside the domain,
// plus sum r^2 and sum b^2 into acc, over half z-rows, with the Laplacian summed in the order
// +x, -x, +y, -y, +z, -z, -6 p. p null: p = 0 (r = b).
// The grid is a few CTAs per SM, each looping over leaf groups and adding its two sums to acc
// once: the FP64 atomics on the two sums serialise in one L2 slice, and one per leaf pair cost
// more than a tenth of the kernel.
__global__ void __launch_bounds__(kThreads) refine_residual_kernel(TopoView t, const float* __restrict__ div,
                                                                    const double* __restrict__ p,
                                                                    float* __restrict__ r, double h2,
                                                                    const double* __restrict__ check, double tol2,
                                                                    double* __restrict__ acc) {
    if (converged(check, tol2)) return;
    double r2 = 0.0, b2 = 0.0;
    const int64_t groups = (t.num_leaves + kRowLeaves - 1) / kRowLeaves;
#pragma unroll 1
    for (int64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        HalfRow w;
        if (!half_row(t, w, g)) continue;
        const float4 d = __ldg(reinterpret_cast<const float4*>(div + w.own));
        const float dv[4] = {d.x, d.y, d.z, d.w};
        double res[4];
        if (p != nullptr) {
            const NbrRows q = nbr_rows(w);
            double c[4], xp[4], xm[4], yp[4], ym[4];
            ld_half4(p + w.own, c);
            ld_half4(p + q.xp, xp);
            ld_half4(p + q.xm, xm);
            ld_half4(p + q.yp, yp);
            ld_half4(p + q.ym, ym);
            int64_t zin_s, zface_s;
            z_ends(w, zin_s, zface_s);
            const double zin = __ldg(p + zin_s), zface = zface_s < 0 ? 0.0 : __ldg(p + zface_s);
            const double zlo = w.h ? zin : zface, zhi = w.h ? zface : zin;
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                const double lap = (q.zxp ? 0.0 : xp[z]) + (q.zxm ? 0.0 : xm[z]) + (q.zyp ? 0.0 : yp[z]) +
                                   (q.zym ? 0.0 : ym[z]) + (z < 3 ? c[z + 1] : zhi) + (z > 0 ? c[z - 1] : zlo) -
                                   6.0 * c[z];
                res[z] = (double)dv[z] * h2 - lap;
            }
        } else {
#pragma unroll
            for (int z = 0; z < 4; ++z) res[z] = (double)dv[z] * h2;
        }
        *reinterpret_cast<float4*>(r + w.own) = make_float4((float)res[0], (float)res[1], (float)res[2], (float)res[3]);
#pragma unroll
        for (int z = 0; z < 4; ++z) {
            const double bb = (double)dv[z] * h2;
            r2 += res[z] * res[z];
            b2 += bb * bb;
        }
    }
    block_sum2(r2, b2, acc);
}

// Slot of the colour-packed layout of the FP16 inner solve (launch_rbgs_packed_half): z of a
// row is stored at position (z & 1) * 4 + (z >> 1).
__device__ __forceinline__ int64_t packed_slot(int64_t q) { return (q & ~int64_t(7)) | ((q & 1) << 2) | ((q >> 1) & 3); }

// Slot of the colour-split layout (launch_rbgs_split_half): a leaf's red values, then its black
// ones; within a colour, the row (x, y) = (a, b) at position R = 32 ((a + b) & 1) + 4 a + (b >> 1),
// entry 4 R + (z >> 1).
__device__ __forceinline__ int64_t split_slot(int64_t q) {
    const int n = (int)(q & 511), a = n >> 6, b = (n >> 3) & 7, z = n & 7;
    const int colour = (a + b + z) & 1;
    const int row = 32 * ((a + b) & 1) + 4 * a + (b >> 1);
    return (q & ~int64_t(511)) | (colour << 8) | (row << 2) | (z >> 1);
}

template <int kLayout>
__device__ __forceinline__ int64_t inner_slot(int64_t q) {
    if constexpr (kLayout == HNS_INNER_PACKED) return packed_slot(q);
    else if constexpr (kLayout == HNS_INNER_SPLIT) return split_slot(q);
    else return q;
}

// r^ = r / s with s = rms(r) from the latest check (stored into *scale); FP16 or FP32;
// r^ in the inner solve's layout kLayout.
template <typename TI, int kLayout>
__global__ void __launch_bounds__(kThreads) refine_scale_kernel(const float* __restrict__ r, TI* __restrict__ rhat,
                                                                 int64_t n, const double* __restrict__ check,
                                                                 double tol2, float* __restrict__ scale) {
    if (converged(check, tol2)) return;
    const double rms = sqrt(check[0] / (double)n);
    const float sc = rms > 0.0 ? (float)rms : 1.0f;
    const float inv = 1.0f / sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) *scale = sc;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        sstore(rhat, inner_slot<kLayout>(q), __ldg(r + q) * inv);
}

// The same for FP16 r^ in the colour-split layout, four slots (half a z-row, z = 4h .. 4h + 3)
// per thread: one 16-byte load and two 4-byte stores, z = 4h and 4h + 2 to entries 2h and 2h + 1
// of the row in one colour, z = 4h + 1 and 4h + 3 to the same entries in the other. The values
// are refine_scale_kernel's to the bit (FP32 product, one FP16 rounding).
__global__ void __launch_bounds__(kThreads) refine_scale_split_kernel(const float* __restrict__ r,
                                                                       __half* __restrict__ rhat, int64_t n,
                                                                       const double* __restrict__ check, double tol2,
                                                                       float* __restrict__ scale) {
    if (converged(check, tol2)) return;
    const double rms = sqrt(check[0] / (double)n);
    const float sc = rms > 0.0 ? (float)rms : 1.0f;
    const float inv = 1.0f / sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) *scale = sc;
    auto h16 = [](float v) { return (uint32_t)__half_as_ushort(__float2half_rn(v)); };
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < (n >> 2); u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = u << 2;
        const float4 v = __ldg(reinterpret_cast<const float4*>(r + q));
        const int loc = (int)(q & 511), a = loc >> 6, b = (loc >> 3) & 7, h = (loc >> 2) & 1;
        const int p0 = (a + b) & 1;
        const int64_t base = (q & ~int64_t(511)) + 4 * (32 * p0 + 4 * a + (b >> 1)) + 2 * h;
        *reinterpret_cast<uint32_t*>(rhat + base + ((int64_t)p0 << 8)) = h16(v.x * inv) | (h16(v.z * inv) << 16);
        *reinterpret_cast<uint32_t*>(rhat + base + ((int64_t)(p0 ^ 1) << 8)) = h16(v.y * inv) | (h16(v.w * inv) << 16);
    }
}

// p += s e (FP64), pointwise; e in the inner solve's layout kLayout. first: the first outer
// iteration, where p = 0 before it: p = 0 + s e without reading p (and p = 0 if the solve had
// converged before any correction), so that p needs no clearing pass.
template <typename TI, int kLayout>
__global__ void __launch_bounds__(kThreads) refine_update_kernel(double* __restrict__ p, const TI* __restrict__ e,
                                                                  int64_t n, const float* __restrict__ scale,
                                                                  const double* __restrict__ check, double tol2,
                                                                  bool first) {
    const int64_t q0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, dq = (int64_t)gridDim.x * blockDim.x;
    if (converged(check, tol2)) {
        if (first)
            for (int64_t q = q0; q < n; q += dq) p[q] = 0.0;
        return;
    }
    const double sc = (double)*scale;
    if (first)
        for (int64_t q = q0; q < n; q += dq) p[q] = 0.0 + sc * (double)sload(e, inner_slot<kLayout>(q));
    else
        for (int64_t q = q0; q < n; q += dq) p[q] += sc * (double)sload(e, inner_slot<kLayout>(q));
}

// The same update from FP16 e in the colour-split layout, four slots per thread (as
// refine_scale_split_kernel): two 4-byte loads of e and 16-byte accesses to p; the values are
// refine_update_kernel's to the bit.
__global__ void __launch_bounds__(kThreads) refine_update_split_kernel(double* __restrict__ p, const __half* __restrict__ e,
                                                                        int64_t n, const float* __restrict__ scale,
                                                                        const double* __restrict__ check, double tol2,
                                                                        bool first) {
    const int64_t u0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, du = (int64_t)gridDim.x * blockDim.x;
    if (converged(check, tol2)) {
        if (first)
            for (int64_t u = u0; u < (n >> 2); u += du) {
                double2* pp = reinterpret_cast<double2*>(p + (u << 2));
                pp[0] = make_double2(0.0, 0.0);
                pp[1] = make_double2(0.0, 0.0);
            }
        return;
    }
    const double sc = (double)*scale;
    auto f = [](uint32_t bits) { return (double)__half2float(__ushort_as_half((unsigned short)bits)); };
    for (int64_t u = u0; u < (n >> 2); u += du) {
        const int64_t q = u << 2;
        const int loc = (int)(q & 511), a = loc >> 6, b = (loc >> 3) & 7, h = (loc >> 2) & 1;
        const int p0 = (a + b) & 1;
        const int64_t base = (q & ~int64_t(511)) + 4 * (32 * p0 + 4 * a + (b >> 1)) + 2 * h;
        const uint32_t w0 = __ldg(reinterpret_cast<const unsigned int*>(e + base + ((int64_t)p0 << 8)));
        const uint32_t w1 = __ldg(reinterpret_cast<const unsigned int*>(e + base + ((int64_t)(p0 ^ 1) << 8)));
        const double d0 = sc * f(w0 & 0xFFFFu), d1 = sc * f(w1 & 0xFFFFu), d2 = sc * f(w0 >> 16), d3 = sc * f(w1 >> 16);
        double2* pp = reinterpret_cast<double2*>(p + q);
        if (first) {
            pp[0] = make_double2(0.0 + d0, 0.0 + d1);
            pp[1] = make_double2(0.0 + d2, 0.0 + d3);
        } else {
            double2 x = pp[0], y = pp[1];
            x.x += d0, x.y += d1, y.x += d2, y.y += d3;
            pp[0] = x;
            pp[1] = y;
        }
    }
}


unsigned row_blocks(const Context& c) { return (unsigned)((c.topo.num_leaves + kRowLeaves - 1) / kRowLeaves); }

// Residual grid: one wave, kResidualCtasPerSm CTAs per SM (the register limit at 62 registers),
// at most one per leaf group. Measured on a 45,198-leaf grid, six refinement residuals per step:
// one CTA per leaf pair 1.35 ms of refinement work outside the inner solves, 6 CTAs per SM 1.28,
// 12 per SM 1.18, 4 per SM 1.15 ms.
constexpr int kResidualCtasPerSm = 4;
unsigned residual_blocks(const Context& c) {
    return std::max(1u, std::min(row_blocks(c), (unsigned)(c.sm_count() * kResidualCtasPerSm)));
}

// Outer iterations the most recent refined solve whose checks have reached the host needed
// (0: unknown), read without waiting: the solve's checks were copied to pinned memory behind
// an event, which is only queried.
int refine_forecast(Context& c) {
    if (!c.refine_echo_pending) return c.refine_forecast;
    const cudaError_t q = cudaEventQuery(c.refine_echo_done);
    if (q == cudaErrorNotReady) return c.refine_forecast;
    HNS_CUDA(q);
    c.refine_echo_pending = false;
    c.refine_forecast = 0;
    const double t2 = c.refine_echo_tol * c.refine_echo_tol;
    for (int k = 1; k <= c.refine_echo_outer; ++k)
        if (c.refine_echo[2 * k] <= t2 * c.refine_echo[2 * k + 1]) {
            c.refine_forecast = k;
            break;
        }
    return c.refine_forecast;
}

// Copies the solve's checks to pinned memory behind an event, for the forecast of later solves.
void refine_echo(Context& c, const RefinePlan& plan) {
    if (2 * (plan.max_outer + 1) > Context::kEchoSlots) return;
    if (c.refine_echo == nullptr) {
        HNS_CUDA(cudaMallocHost(&c.refine_echo, sizeof(double) * Context::kEchoSlots));
        HNS_CUDA(cudaEventCreateWithFlags(&c.refine_echo_done, cudaEventDisableTiming));
    }
    HNS_CUDA(cudaMemcpyAsync(c.refine_echo, plan.slots, sizeof(double) * 2 * (size_t)(plan.max_outer + 1),
                             cudaMemcpyDeviceToHost, c.stream));
    HNS_CUDA(cudaEventRecord(c.refine_echo_done, c.stream));
    c.refine_echo_pending = true;
    c.refine_echo_outer = plan.max_outer;
    c.refine_echo_tol = plan.tol;
}

bool capturing(const Context& c) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    HNS_CUDA(cudaStreamIsCapturing(c.stream, &st));
    return st != cudaStreamCaptureStatusNone;
}

// Condition of a spare outer iteration's graph: 1 while the refinement has not converged (the
// test every kernel of the iteration makes before it does anything).
__global__ void spare_gate_kernel(cudaGraphConditionalHandle h, const double* __restrict__ check, double tol2) {
    cudaGraphSetConditional(h, check[0] <= tol2 * check[1] ? 0u : 1u);
}

// Runs `body` (the launches of one outer iteration whose kernels return at once after
// convergence) on the stream as a graph whose conditional node skips it on the device after
// convergence: one gate kernel and a graph launch in place of the iteration's launches. The
// graph is made on the first call with this key (body captured once) and relaunched after.
// Returns false, with nothing enqueued, where a graph cannot be made.
bool run_spare_graph(Context& c, const std::vector<uintptr_t>& key, const double* check, double tol2,
                     const std::function<void()>& body) {
    if (c.spare_graph_ok == 0) return false;
    Context::SpareGraph* found = nullptr;
    for (auto& g : c.spare_graphs)
        if (g.key == key) found = &g;
    if (found == nullptr) {
        if (c.spare_graphs.size() >= 16) c.release_spare_graphs();
        Context::SpareGraph sg;
        sg.key = key;
        bool ok = cudaGraphCreate(&sg.graph, 0) == cudaSuccess;
        cudaGraphConditionalHandle h = 0;
        cudaGraph_t body_graph = nullptr;
        cudaGraphNode_t gate = nullptr, cond = nullptr;
        if (ok) ok = cudaGraphConditionalHandleCreate(&h, sg.graph, 0, 0) == cudaSuccess;
        if (ok) {
            cudaKernelNodeParams kp = {};
            void* args[] = {&h, &check, &tol2};
            kp.func = reinterpret_cast<void*>(spare_gate_kernel);
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(1);
            kp.kernelParams = args;
            ok = cudaGraphAddKernelNode(&gate, sg.graph, nullptr, 0, &kp) == cudaSuccess;
        }
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&cond, sg.graph, &gate, 1, &cp) == cudaSuccess;
            if (ok) body_graph = cp.conditional.phGraph_out[0];
        }
        if (ok) {
            // The body's launches are captured, not run; no phase events inside the graph.
            const bool prof = c.profiling;
            c.profiling = false;
            ok = cudaStreamBeginCaptureToGraph(c.stream, body_graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
                 cudaSuccess;
            if (ok) {
                try {
                    body();
                } catch (const Error&) {
                    ok = false;
                }
                cudaGraph_t out = nullptr;
                if (cudaStreamEndCapture(c.stream, &out) != cudaSuccess) ok = false;
            }
            c.profiling = prof;
        }
        if (ok) ok = cudaGraphInstantiate(&sg.exec, sg.graph, 0) == cudaSuccess;
        if (!ok) {
            (void)cudaGetLastError();
            if (sg.exec) (void)cudaGraphExecDestroy(sg.exec);
            if (sg.graph) (void)cudaGraphDestroy(sg.graph);
            c.spare_graph_ok = 0;
            return false;
        }
        c.spare_graph_ok = 1;
        c.spare_graphs.push_back(sg);
        found = &c.spare_graphs.back();
    }
    HNS_CUDA(cudaGraphLaunch(found->exec, c.stream));
    HNS_LAUNCHED();  // the gate kernel
    return true;
}

// Grid of the grid-stride passes: four values per thread, at most 32 CTAs per SM.
unsigned stream_blocks(const Context& c, int64_t n) {
    const int64_t b = (n + kThreads * 4 - 1) / (kThreads * 4);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)c.sm_count() * 32));
}

// ---- conversions -------------------------------------------------------------------------

template <typename D, typename Src>
__global__ void convert_kernel(const Src* __restrict__ src, D* __restrict__ dst, int64_t n);

template <>
__global__ void convert_kernel<__nv_bfloat16, float>(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = __float2bfloat16_rn(src[q]);
}
template <>
__global__ void convert_kernel<float, __nv_bfloat16>(const __nv_bfloat16* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = __bfloat162float(src[q]);
}
template <>
__global__ void convert_kernel<__half, float>(const float* __restrict__ src, __half* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = __float2half_rn(src[q]);
}
template <>
__global__ void convert_kernel<float, __half>(const __half* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = __half2float(src[q]);
}
template <>
__global__ void convert_kernel<double, float>(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = (double)src[q];
}
template <>
__global__ void convert_kernel<float, double>(const double* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dst[q] = (float)src[q];
}

size_t dtype_size(int dt) {
    switch (dt) {
        case HNS_DTYPE_F32: return 4;
        case HNS_DTYPE_F16: return 2;
        case HNS_DTYPE_BF16: return 2;
        case HNS_DTYPE_F64: return 8;
    }
    fail(HNS_ERR_INVALID_ARG, "unknown dtype");
}

}  // namespace

void convert_array(const Context& c, const void* src, int src_dt, void* dst, int dst_dt, int64_t n) {
    if (n <= 0) return;
    const unsigned g = stream_blocks(c, n);
    if (src_dt == dst_dt) {
        HNS_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * dtype_size(src_dt), cudaMemcpyDeviceToDevice, c.stream));
        return;
    }
    if (src_dt == HNS_DTYPE_F32 && dst_dt == HNS_DTYPE_BF16)
        convert_kernel<__nv_bfloat16, float><<<g, kThreads, 0, c.stream>>>((const float*)src, (__nv_bfloat16*)dst, n);
    else if (src_dt == HNS_DTYPE_BF16 && dst_dt == HNS_DTYPE_F32)
        convert_kernel<float, __nv_bfloat16><<<g, kThreads, 0, c.stream>>>((const __nv_bfloat16*)src, (float*)dst, n);
    else if (src_dt == HNS_DTYPE_F32 && dst_dt == HNS_DTYPE_F16)
        convert_kernel<__half, float><<<g, kThreads, 0, c.stream>>>((const float*)src, (__half*)dst, n);
    else if (src_dt == HNS_DTYPE_F16 && dst_dt == HNS_DTYPE_F32)
        convert_kernel<float, __half><<<g, kThreads, 0, c.stream>>>((const __half*)src, (float*)dst, n);
    else if (src_dt == HNS_DTYPE_F32 && dst_dt == HNS_DTYPE_F64)
        convert_kernel<double, float><<<g, kThreads, 0, c.stream>>>((const float*)src, (double*)dst, n);
    else if (src_dt == HNS_DTYPE_F64 && dst_dt == HNS_DTYPE_F32)
        convert_kernel<float, double><<<g, kThreads, 0, c.stream>>>((const double*)src, (float*)dst, n);
    else
        fail(HNS_ERR_UNSUPPORTED, "conversion between these dtypes is not provided");
    HNS_LAUNCHED();
}

// Refinement loop: enqueues `max_outer` outer iterations of `inner` red-black iterations each
// (inner storage TI), stopping on the device at ||r|| <= tol ||b||. p (FP64, n values) is
// overwritten. Returns the schedule for refine_result().
template <typename TI>
RefinePlan refine_solve(Context& c, const float* div, double* p, int max_outer, int inner, float omega, double tol,
                        unsigned flags) {
    if (flags & HNS_SOLVE_NEUMANN)
        fail(HNS_ERR_UNSUPPORTED, "zero-gradient walls are supported by the plain red-black solve only");
    const int64_t n = c.num_voxels();
    RefinePlan plan;
    plan.max_outer = std::max(1, max_outer);
    plan.inner = std::max(1, inner);
    plan.tol = tol;
    plan.inner_fp16 = sizeof(TI) == 2;
    const int slots_needed = 8 + 2 * (plan.max_outer + 1) + plan.max_outer;
    double* base = c.reduce_slots(slots_needed);
    plan.slots = base + 8;
    float* scales = reinterpret_cast<float*>(plan.slots + 2 * (plan.max_outer + 1));
    HNS_CUDA(cudaMemsetAsync(plan.slots, 0, sizeof(double) * (size_t)(2 * (plan.max_outer + 1) + plan.max_outer), c.stream));
    float* r = c.scratch_f32("refine_r", (size_t)n);
    TI* rhat = reinterpret_cast<TI*>(c.scratch_f32("refine_rhat", ((size_t)n * sizeof(TI) + 3) / 4));
    TI* e[2] = {reinterpret_cast<TI*>(c.scratch_f32("refine_e0", ((size_t)n * sizeof(TI) + 3) / 4)),
                reinterpret_cast<TI*>(c.scratch_f32("refine_e1", ((size_t)n * sizeof(TI) + 3) / 4))};
    const double h2 = (double)c.dx * (double)c.dx;
    const double tol2 = tol * tol;
    const unsigned g = stream_blocks(c, n);
    // The FP16 inner solve's layout is an option (colour-split, colour-packed or plain order); the
    // FP32 inner solve takes the colour-split layout with the colour-split FP32 kernel.
    const int layout = sizeof(TI) == 2 ? c.inner_layout
                                       : (c.rbgs_kernel == HNS_RBGS_SPLIT ? HNS_INNER_SPLIT : HNS_INNER_ROWS);
    const bool packed = layout == HNS_INNER_PACKED;
    // Colour-split: e in place with one extra all-zero leaf, and the face-neighbour table (both
    // depend on the topology alone: made once per buffer).
    TI* e_split = nullptr;
    int* nb8 = nullptr;
    if (layout == HNS_INNER_SPLIT) {
        e_split = sizeof(TI) == 2 ? static_cast<TI*>(c.split_e("refine_e_split", sizeof(TI), 0))
                                  : static_cast<TI*>(c.split_e("refine_e_split32", sizeof(TI), 2));
        nb8 = c.split_faces();
    }
    // HNS_OPT_L2_PERSIST: the FP16 colour-split correction array persisting in L2 for this solve's
    // inner launches (their access-policy window), reset when the solve has been enqueued; only
    // where the whole array fits the device's persisting-L2 maximum. Measured: shell512 (46 MB)
    // 3.59 -> 3.55 ms per step; fire1024 (191 MB against 79 MB, hit ratio 0.41) 20.0 -> 26.1 ms,
    // its persisting lines slowing the other phases too.
    struct WindowReset {
        Context& c;
        ~WindowReset() { c.inner_window = {}; }
    } window_reset{c};
    if (c.l2_persist && sizeof(TI) == 2 && e_split != nullptr) {
        int max_window = 0, max_persist = 0;
        HNS_CUDA(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, c.device));
        HNS_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, c.device));
        const size_t bytes = (size_t)n * sizeof(TI);
        const size_t persist = bytes;
        // Not while the caller captures the stream before this context has raised the limit (a
        // device-wide call inside a capture).
        if (bytes > 0 && bytes <= (size_t)std::max(0, max_window) && bytes <= (size_t)std::max(0, max_persist) &&
            (c.l2_persist_limit >= persist || !capturing(c))) {
            if (c.l2_persist_limit < persist) c.l2_persist_limit = raise_device_setting(c.device, 1, persist);
            c.inner_window.base_ptr = e_split;
            c.inner_window.num_bytes = bytes;
            c.inner_window.hitRatio = 1.0f;
            c.inner_window.hitProp = cudaAccessPropertyPersisting;
            c.inner_window.missProp = cudaAccessPropertyStreaming;
        }
    }
    // Packed: the face buffers of e[0] and e[1] and the rhs halo records.
    void* faces[2] = {nullptr, nullptr};
    void* halo = nullptr;
    if (packed) {
        const size_t leaves = (size_t)c.topo.num_leaves;
        faces[0] = c.scratch_f32("refine_faces0", leaves * kPackedFaceBytes / 4);
        faces[1] = c.scratch_f32("refine_faces1", leaves * kPackedFaceBytes / 4);
        halo = c.scratch_f32("refine_rhs_halo", leaves * kPackedHaloBytes / 4);
    }
    // r = b; p is written by the first update (refine_update_kernel with first set).
    refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, div, nullptr, r, h2, nullptr,
                                                                         tol2, plan.slots);
    HNS_LAUNCHED();
    // Outer iterations past the forecast launch on short grids (one wave, looping): if the
    // refinement has converged they return at once for the cost of the launch alone.
    const bool echo = !capturing(c);
    const int forecast = echo ? refine_forecast(c) : 0;
    // Multigrid on the FP16 colour-split layout: `inner` V-cycles per outer iteration, the
    // colour-split half-sweep as the fine smoother (mg16_vcycle); other layouts and the FP32
    // inner solve take the FP32 V-cycle in slot order below.
    const bool mg16 = (flags & HNS_SOLVE_MULTIGRID) && sizeof(TI) == 2 && layout == HNS_INNER_SPLIT;
    auto mg16_iteration = [&](int k, unsigned gk) {
        const double* chk = plan.slots + 2 * k;
        refine_scale_split_kernel<<<gk, kThreads, 0, c.stream>>>(r, reinterpret_cast<__half*>(rhat), n, chk, tol2,
                                                                 scales + k);
        HNS_LAUNCHED();
        c.phase_begin(HNS_PHASE_INNER);
        for (int cyc = 0; cyc < plan.inner; ++cyc) mg16_vcycle(c, nb8, rhat, e_split, cyc == 0, chk, tol2);
        c.phase_end();
        refine_update_split_kernel<<<gk, kThreads, 0, c.stream>>>(p, reinterpret_cast<const __half*>(e_split), n,
                                                                  scales + k, chk, tol2, k == 0);
        HNS_LAUNCHED();
        refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, div, p, r, h2, chk, tol2,
                                                                             plan.slots + 2 * (k + 1));
        HNS_LAUNCHED();
    };
    for (int k = 0; k < plan.max_outer; ++k) {
        const double* chk = plan.slots + 2 * k;
        const bool spare = forecast > 0 && k >= forecast;
        const unsigned gk = spare ? std::min(g, (unsigned)(c.sm_count() * 4)) : g;
        if (mg16) {
            // Past the forecast, the iteration most likely finds the solve converged: as a graph
            // whose device-side condition skips it then (one gate kernel in place of 65 or more
            // returning launches), else launched as the others.
            if (spare) {
                uint64_t tol_bits = 0;
                std::memcpy(&tol_bits, &tol2, sizeof tol_bits);
                const std::vector<uintptr_t> key = {
                    (uintptr_t)k, (uintptr_t)gk, (uintptr_t)plan.inner, (uintptr_t)p, (uintptr_t)div, (uintptr_t)r,
                    (uintptr_t)rhat, (uintptr_t)e_split, (uintptr_t)nb8, (uintptr_t)plan.slots, (uintptr_t)scales,
                    (uintptr_t)plan.max_outer, (uintptr_t)n,
                    (uintptr_t)c.coarse_solve, (uintptr_t)c.coarse_cluster_ok, (uintptr_t)c.split_solve,
                    (uintptr_t)c.first_wait_polls, (uintptr_t)c.inner_window.num_bytes, (uintptr_t)tol_bits};
                if (run_spare_graph(c, key, chk, tol2, [&] { mg16_iteration(k, gk); })) continue;
            }
            mg16_iteration(k, gk);
            continue;
        }
        if ((flags & HNS_SOLVE_MULTIGRID) && !mg16) {
            // One V-cycle on the scaled residual in FP32 (slot order), then p += s e.
            float* rm = c.scratch_f32("mg_rhat", (size_t)n);
            float* em = c.scratch_f32("mg_e", (size_t)n);
            refine_scale_kernel<float, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(r, rm, n, chk, tol2, scales + k);
            HNS_LAUNCHED();
            c.phase_begin(HNS_PHASE_INNER);
            mg_vcycle(c, rm, em, chk, tol2);
            c.phase_end();
            refine_update_kernel<float, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(p, em, n, scales + k, chk, tol2,
                                                                                       k == 0);
            HNS_LAUNCHED();
            refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, div, p, r, h2, chk, tol2, plan.slots + 2 * (k + 1));
            HNS_LAUNCHED();
            continue;
        }
        if (layout == HNS_INNER_PACKED)
            refine_scale_kernel<TI, HNS_INNER_PACKED><<<gk, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        else if (layout == HNS_INNER_SPLIT) {
            if constexpr (sizeof(TI) == 2)
                refine_scale_split_kernel<<<gk, kThreads, 0, c.stream>>>(r, reinterpret_cast<__half*>(rhat), n, chk, tol2,
                                                                         scales + k);
            else
                refine_scale_kernel<TI, HNS_INNER_SPLIT><<<gk, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        } else
            refine_scale_kernel<TI, HNS_INNER_ROWS><<<gk, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        HNS_LAUNCHED();
        if (packed) launch_rhs_halo_pack(c, rhat, halo, chk, tol2);
        const TI* src = nullptr;
        const void* src_faces = nullptr;
        c.phase_begin(HNS_PHASE_INNER);
        // The persistent form: the whole inner solve in one launch. An outer iteration past the
        // forecast takes it whatever the option: it most likely returns at once, and one launch
        // then costs a few microseconds where 2 * inner returning half-sweeps cost 2.3 us each.
        const bool persistent = layout == HNS_INNER_SPLIT && (c.split_solve == HNS_SPLIT_PERSISTENT || spare);
        if (persistent) {
            if constexpr (sizeof(TI) == 2)
                launch_rbgs_split_solve(c, nb8, rhat, e_split, 2 * plan.inner, true, omega, chk, tol2);
            else
                launch_rbgs_split_solve_f32(c, nb8, reinterpret_cast<const float*>(rhat), reinterpret_cast<float*>(e_split),
                                            2 * plan.inner, true, omega, 1.0f, chk, tol2);
            src = e_split;
        }
        for (int it = 0; it < (persistent ? 0 : plan.inner); ++it) {
            TI* dst = e[it & 1];
            if constexpr (sizeof(TI) == 2) {
                if (layout == HNS_INNER_SPLIT) {
                    // In place: red, then black.
                    dst = e_split;
                    launch_rbgs_split_half(c, nb8, rhat, dst, 0, it == 0, omega, chk, tol2, spare);
                    launch_rbgs_split_half(c, nb8, rhat, dst, 1, false, omega, chk, tol2, spare);
                } else if (packed) {
                    launch_rbgs_packed_half(c, rhat, halo, src, src_faces, dst, faces[it & 1], omega, chk, tol2);
                    src_faces = faces[it & 1];
                } else
                    launch_rbgs_bulk_half(c, rhat, src, dst, omega, chk, tol2);
            } else if (layout == HNS_INNER_SPLIT) {
                // In place on the FP32 colour-split e: red, then black (unit dx^2).
                dst = e_split;
                auto* ef = reinterpret_cast<float*>(dst);
                const auto* rf = reinterpret_cast<const float*>(rhat);
                launch_rbgs_split_half_f32(c, nb8, rf, ef, 0, it == 0, omega, 1.0f, chk, tol2, spare);
                launch_rbgs_split_half_f32(c, nb8, rf, ef, 1, false, omega, 1.0f, chk, tol2, spare);
            } else
                launch_rbgs_bulk_unit(c, reinterpret_cast<const float*>(rhat), reinterpret_cast<const float*>(src),
                                      reinterpret_cast<float*>(dst), omega, chk, tol2);
            src = dst;
        }
        c.phase_end();
        if (layout == HNS_INNER_PACKED)
            refine_update_kernel<TI, HNS_INNER_PACKED><<<gk, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2, k == 0);
        else if (layout == HNS_INNER_SPLIT) {
            if constexpr (sizeof(TI) == 2)
                refine_update_split_kernel<<<gk, kThreads, 0, c.stream>>>(p, reinterpret_cast<const __half*>(src), n,
                                                                          scales + k, chk, tol2, k == 0);
            else
                refine_update_kernel<TI, HNS_INNER_SPLIT><<<gk, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2,
                                                                                          k == 0);
        } else
            refine_update_kernel<TI, HNS_INNER_ROWS><<<gk, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2, k == 0);
        HNS_LAUNCHED();
        refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, div, p, r, h2, chk, tol2, plan.slots + 2 * (k + 1));
        HNS_LAUNCHED();
    }
    if (echo) refine_echo(c, plan);
    log_solve(c, plan.slots, plan.max_outer + 1, tol, plan.inner, 0, plan.max_outer * plan.inner);
    return plan;
}

template RefinePlan refine_solve<__half>(Context&, const float*, double*, int, int, float, double, unsigned);
template RefinePlan refine_solve<float>(Context&, const float*, double*, int, int, float, double, unsigned);

void refine_result(Context& c, const RefinePlan& plan, int* outer, double* residual) {
    std::vector<double> h(2 * (size_t)(plan.max_outer + 1));
    HNS_CUDA(cudaMemcpyAsync(h.data(), plan.slots, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    HNS_CUDA(cudaStreamSynchronize(c.stream));
    const double tol2 = plan.tol * plan.tol;
    for (int k = 0; k <= plan.max_outer; ++k) {
        if (h[2 * k] <= tol2 * h[2 * k + 1] || k == plan.max_outer) {
            *outer = k;
            *residual = h[2 * k + 1] > 0 ? std::sqrt(h[2 * k] / h[2 * k + 1]) : 0.0;
            return;
        }
    }
}

namespace {

// Voxel records for the mixed advection: a voxel's BF16 velocity and its first FP16 scalar as
// one 8-byte record (u | v << 16, w | s << 16), so that each of the 2 x 8 trace taps and 6 clamp
// neighbours is one load instead of four. Four voxels per thread: three 8-byte loads of
// velocity, one of the scalar, two 16-byte stores.
__global__ void __launch_bounds__(kThreads) pack_records_kernel(const __nv_bfloat16* __restrict__ vel,
                                                                 const __half* __restrict__ s0, uint4* __restrict__ rec,
                                                                 int64_t n) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < (n >> 2); u += (int64_t)gridDim.x * blockDim.x) {
        const uint2* pv = reinterpret_cast<const uint2*>(vel + 12 * u);
        const uint2 a = __ldg(pv), b = __ldg(pv + 1), c = __ldg(pv + 2);
        const uint2 d = s0 != nullptr ? __ldg(reinterpret_cast<const uint2*>(s0 + 4 * u)) : make_uint2(0u, 0u);
        rec[2 * u] = make_uint4(a.x, (a.y & 0xFFFFu) | (d.x << 16), (a.y >> 16) | (b.x << 16), (b.x >> 16) | (d.x & 0xFFFF0000u));
        rec[2 * u + 1] = make_uint4(b.y, (c.x & 0xFFFFu) | (d.y << 16), (c.x >> 16) | (c.y << 16), (c.y >> 16) | (d.y & 0xFFFF0000u));
    }
}

// The record at slot s (-1: outside the domain, all zero), as FP32 velocity and scalar.
struct Rec {
    float u, v, w, d;
};
__device__ __forceinline__ Rec rec_at(const uint2* __restrict__ rec, int32_t s) {
    if (s < 0) return Rec{0.f, 0.f, 0.f, 0.f};
    const uint2 r = __ldg(rec + (uint32_t)s);
    return Rec{__uint_as_float(r.x << 16), __uint_as_float(r.x & 0xFFFF0000u), __uint_as_float(r.y << 16),
               __half2float(__ushort_as_half((unsigned short)(r.y >> 16)))};
}

// advect_mixed_kernel on voxel records: the same trace, taps, lerps and clamps in the same
// order, so the same bits; the velocity and the first scalar come from the records, further
// scalars (f) from their own arrays. 32-bit slots (fewer than 2^22 leaves).
__global__ void __launch_bounds__(kThreads, 4) advect_records_kernel(TopoView t, const uint2* __restrict__ rec,
                                                                      __nv_bfloat16* __restrict__ vel_out,
                                                                      __half* __restrict__ s0_out, FieldSetT<__half> f,
                                                                      float sdt) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int32_t s = (int32_t(v.leaf) << 9) + int32_t(v.n);
    const Rec o = rec_at(rec, s);
    const float bx = (float)i - o.u * sdt, by = (float)j - o.v * sdt, bz = (float)k - o.w * sdt;
    TapsT<int32_t> tb, tf;
    taps_at(tb, t, L, bx, by, bz);
    float x[8], y[8], z[8], d[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const Rec a = rec_at(rec, tb.s[q]);
        x[q] = a.u, y[q] = a.v, z[q] = a.w, d[q] = a.d;
    }
    const float3 vf = make_float3(tri_lerp(tb, x), tri_lerp(tb, y), tri_lerp(tb, z));
    const float pf = tri_lerp(tb, d);
    taps_at(tf, t, L, bx + vf.x * sdt, by + vf.y * sdt, bz + vf.z * sdt);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const Rec a = rec_at(rec, tf.s[q]);
        x[q] = a.u, y[q] = a.v, z[q] = a.w, d[q] = a.d;
    }
    const float3 vb = make_float3(tri_lerp(tf, x), tri_lerp(tf, y), tri_lerp(tf, z));
    const float pb = tri_lerp(tf, d);
    int32_t ns[6];
    face_slots(L, s, v.n, ns);
    float3 corr = make_float3(vf.x + 0.5f * (o.u - vb.x), vf.y + 0.5f * (o.v - vb.y), vf.z + 0.5f * (o.w - vb.z));
    float3 mn = make_float3(o.u, o.v, o.w), mx = mn;
    float dmn = o.d, dmx = o.d;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const Rec a = rec_at(rec, ns[q]);
        mn.x = fminf(mn.x, a.u), mn.y = fminf(mn.y, a.v), mn.z = fminf(mn.z, a.w);
        mx.x = fmaxf(mx.x, a.u), mx.y = fmaxf(mx.y, a.v), mx.z = fmaxf(mx.z, a.w);
        dmn = fminf(dmn, a.d);
        dmx = fmaxf(dmx, a.d);
    }
    mn.x = fminf(mn.x, vf.x), mn.y = fminf(mn.y, vf.y), mn.z = fminf(mn.z, vf.z);
    mx.x = fmaxf(mx.x, vf.x), mx.y = fmaxf(mx.y, vf.y), mx.z = fmaxf(mx.z, vf.z);
    corr.x = fmaxf(mn.x, fminf(corr.x, mx.x));
    corr.y = fmaxf(mn.y, fminf(corr.y, mx.y));
    corr.z = fmaxf(mn.z, fminf(corr.z, mx.z));
    if (vel_out != nullptr) vstore(vel_out, wide(s), corr);
    if (s0_out != nullptr) {
        const float dcorr = pf + 0.5f * (o.d - pb);
        dmn = fminf(dmn, pf);
        dmx = fmaxf(dmx, pf);
        sstore(s0_out, wide(s), fmaxf(dmn, fminf(dcorr, dmx)));
    }
    for (int c = 0; c < f.count; ++c) {
        const __half* __restrict__ dd = f.in[c];
        const float po = sload(dd, wide(s));
        const float qf = tri1(tb, dd);
        const float qb = tri1(tf, dd);
        const float cc = qf + 0.5f * (po - qb);
        float lo = po, hi = po;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float a = tap1(dd, ns[q]);
            lo = fminf(lo, a);
            hi = fmaxf(hi, a);
        }
        lo = fminf(lo, qf);
        hi = fmaxf(hi, qf);
        sstore(f.out[c], wide(s), fmaxf(lo, fminf(cc, hi)));
    }
}

// ---- advection from a leaf tile in shared memory --------------------------------------------
// The advection of the velocity and at most one scalar (advect_records_kernel's arithmetic)
// with the leaf's voxels and a kTileHalo-voxel halo around it read once from the BF16 velocity
// and FP16 scalar arrays into shared memory as FP32 (u, v, w, s), a tile of kTileSide^3 cells
// at local coordinates [-kTileHalo, 8 + kTileHalo), with no record-packing pass. A trace cell
// whose eight corners lie in the tile is eight shared-memory loads at fixed offsets from one
// base index (a back trace shorter than a voxel per axis, and a forward trace that ends within
// a voxel of the start); other cells take the leaf-table path, reading the arrays. The clamp's
// six face neighbours always lie in the tile. Same values, same lerps in the same order, same
// clamps: the records kernel's results to the bit. One CTA of 256 threads per leaf, two voxels
// per thread (x and x + 4), four CTAs per SM so that one CTA's tile fill overlaps the others'
// sampling; cells of missing leaves hold 0, as the records kernel reads outside the domain.
//
// Tile layout: cell (x, y, z) at x * kTileSX + y * kTileSY + z, both strides multiples of 8 cells
// (16-byte cells): the 8 lanes of a quarter-warp, one z-row of voxels, then read cells whose
// bank group is set by z alone, so a row whose traces straddle a y or x cell boundary still
// reads distinct bank groups (an unpadded 10-cell stride measured 38 % bank conflicts).
constexpr int kTileHalo = 1;
constexpr int kTileSide = 8 + 2 * kTileHalo;
constexpr int kTileSY = 16, kTileSX = kTileSide * kTileSY;
constexpr int kTileCells = kTileSide * kTileSide * kTileSide;  // cells filled
constexpr int kTileStore = kTileSide * kTileSX;                // cells allocated (padding included)
constexpr int kTileThreads = 256;
constexpr int kTileFill = (kTileCells + kTileThreads - 1) / kTileThreads;  // cells a thread fills

// Trilinear sample of the four channels at (x, y, z) (global voxel units), lerps along z, then
// y, then x (tri_lerp's order).
// The FP32 (u, v, w, s) of the voxel at slot s from the BF16 velocity and FP16 scalar arrays
// (s0 null: s = 0).
__device__ __forceinline__ float4 voxel4(const __nv_bfloat16* __restrict__ vel, const __half* __restrict__ s0, uint32_t s) {
    const unsigned short* v = reinterpret_cast<const unsigned short*>(vel) + 3 * (size_t)s;
    return make_float4(__uint_as_float((uint32_t)__ldg(v) << 16), __uint_as_float((uint32_t)__ldg(v + 1) << 16),
                       __uint_as_float((uint32_t)__ldg(v + 2) << 16), s0 != nullptr ? __half2float(__ldg(s0 + s)) : 0.f);
}

__device__ __forceinline__ float4 tile_sample(const float4* __restrict__ tile, const TopoView& t, const LeafNbhd& L,
                                              const __nv_bfloat16* __restrict__ vel, const __half* __restrict__ s0,
                                              float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
    const int cx = i - (L.lx << 3) + kTileHalo, cy = j - (L.ly << 3) + kTileHalo, cz = k - (L.lz << 3) + kTileHalo;
    float4 c[8];
    if ((unsigned)cx <= (unsigned)(kTileSide - 2) && (unsigned)cy <= (unsigned)(kTileSide - 2) &&
        (unsigned)cz <= (unsigned)(kTileSide - 2)) {
        const float4* b = tile + cx * kTileSX + cy * kTileSY + cz;
#pragma unroll
        for (int q = 0; q < 8; ++q) c[q] = b[(q >> 2) * kTileSX + ((q >> 1) & 1) * kTileSY + (q & 1)];
    } else {
        TapsT<int32_t> tp;
        taps_at(tp, t, L, x, y, z);
#pragma unroll
        for (int q = 0; q < 8; ++q) c[q] = tp.s[q] < 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : voxel4(vel, s0, (uint32_t)tp.s[q]);
    }
    auto tri = [&](float v0, float v1, float v2, float v3, float v4, float v5, float v6, float v7) {
        const float z0 = lerp1(v0, v1, tz), z1 = lerp1(v2, v3, tz), z2 = lerp1(v4, v5, tz), z3 = lerp1(v6, v7, tz);
        return lerp1(lerp1(z0, z1, ty), lerp1(z2, z3, ty), tx);
    };
    return make_float4(tri(c[0].x, c[1].x, c[2].x, c[3].x, c[4].x, c[5].x, c[6].x, c[7].x),
                       tri(c[0].y, c[1].y, c[2].y, c[3].y, c[4].y, c[5].y, c[6].y, c[7].y),
                       tri(c[0].z, c[1].z, c[2].z, c[3].z, c[4].z, c[5].z, c[6].z, c[7].z),
                       tri(c[0].w, c[1].w, c[2].w, c[3].w, c[4].w, c[5].w, c[6].w, c[7].w));
}

__global__ void __launch_bounds__(kTileThreads, 4) advect_tile_kernel(TopoView t, const __nv_bfloat16* __restrict__ vel,
                                                                       const __half* __restrict__ s0,
                                                                       __nv_bfloat16* __restrict__ vel_out,
                                                                       __half* __restrict__ s0_out, float sdt) {
    __shared__ float4 tile[kTileStore];
    __shared__ LeafNbhd L;
    const int64_t leaf = blockIdx.x;
    load_nbhd(L, t, leaf);
    __syncthreads();
    // The fill: every load of the thread's cells is issued before any is unpacked.
    const unsigned short* vb = reinterpret_cast<const unsigned short*>(vel);
    const unsigned short* sb = reinterpret_cast<const unsigned short*>(s0);
    uint32_t raw[kTileFill][4];
#pragma unroll
    for (int m = 0; m < kTileFill; ++m) {
        const int q = threadIdx.x + m * kTileThreads;
        raw[m][0] = raw[m][1] = raw[m][2] = raw[m][3] = 0u;
        if (q < kTileCells) {
            const int lx = q / (kTileSide * kTileSide) - kTileHalo, ly = (q / kTileSide) % kTileSide - kTileHalo,
                      lz = q % kTileSide - kTileHalo;
            const int r = (lx < 0 ? 0 : lx > 7 ? 18 : 9) + (ly < 0 ? 0 : ly > 7 ? 6 : 3) + (lz < 0 ? 0 : lz > 7 ? 2 : 1);
            const int l = L.nb[r];
            if (l >= 0) {
                const uint32_t sl = ((uint32_t)l << 9) | (uint32_t)(((lx & 7) << 6) | ((ly & 7) << 3) | (lz & 7));
                raw[m][0] = __ldg(vb + 3 * (size_t)sl);
                raw[m][1] = __ldg(vb + 3 * (size_t)sl + 1);
                raw[m][2] = __ldg(vb + 3 * (size_t)sl + 2);
                if (sb != nullptr) raw[m][3] = __ldg(sb + sl);
            }
        }
    }
#pragma unroll
    for (int m = 0; m < kTileFill; ++m) {
        const int q = threadIdx.x + m * kTileThreads;
        if (q < kTileCells) {
            const int at = (q / (kTileSide * kTileSide)) * kTileSX + ((q / kTileSide) % kTileSide) * kTileSY + q % kTileSide;
            tile[at] = make_float4(__uint_as_float(raw[m][0] << 16), __uint_as_float(raw[m][1] << 16),
                                   __uint_as_float(raw[m][2] << 16), __half2float(__ushort_as_half((unsigned short)raw[m][3])));
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
        const int n = (int)threadIdx.x + half * kTileThreads;
        const int a = n >> 6, b = (n >> 3) & 7, cz = n & 7;
        const int i = (L.lx << 3) + a, j = (L.ly << 3) + b, k = (L.lz << 3) + cz;
        const float4* centre = tile + (a + kTileHalo) * kTileSX + (b + kTileHalo) * kTileSY + (cz + kTileHalo);
        const float4 o = *centre;
        const float bx = (float)i - o.x * sdt, by = (float)j - o.y * sdt, bz = (float)k - o.z * sdt;
        const float4 f = tile_sample(tile, t, L, vel, s0, bx, by, bz);
        const float4 g = tile_sample(tile, t, L, vel, s0, bx + f.x * sdt, by + f.y * sdt, bz + f.z * sdt);
        float3 corr = make_float3(f.x + 0.5f * (o.x - g.x), f.y + 0.5f * (o.y - g.y), f.z + 0.5f * (o.z - g.z));
        float3 mn = make_float3(o.x, o.y, o.z), mx = mn;
        float dmn = o.w, dmx = o.w;
        constexpr int kOff[6] = {-kTileSX, kTileSX, -kTileSY, kTileSY, -1, 1};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float4 e = centre[kOff[q]];
            mn.x = fminf(mn.x, e.x), mn.y = fminf(mn.y, e.y), mn.z = fminf(mn.z, e.z);
            mx.x = fmaxf(mx.x, e.x), mx.y = fmaxf(mx.y, e.y), mx.z = fmaxf(mx.z, e.z);
            dmn = fminf(dmn, e.w);
            dmx = fmaxf(dmx, e.w);
        }
        mn.x = fminf(mn.x, f.x), mn.y = fminf(mn.y, f.y), mn.z = fminf(mn.z, f.z);
        mx.x = fmaxf(mx.x, f.x), mx.y = fmaxf(mx.y, f.y), mx.z = fmaxf(mx.z, f.z);
        corr.x = fmaxf(mn.x, fminf(corr.x, mx.x));
        corr.y = fmaxf(mn.y, fminf(corr.y, mx.y));
        corr.z = fmaxf(mn.z, fminf(corr.z, mx.z));
        const int64_t s = (leaf << 9) + n;
        if (vel_out != nullptr) vstore(vel_out, s, corr);
        if (s0_out != nullptr) {
            const float dcorr = f.w + 0.5f * (o.w - g.w);
            dmn = fminf(dmn, f.w);
            dmx = fmaxf(dmx, f.w);
            sstore(s0_out, s, fmaxf(dmn, fminf(dcorr, dmx)));
        }
    }
}

}  // namespace

void launch_advect_mixed(Context& c, const void* vel, void* vel_out, const void* const* sin, void* const* sout, int ns,
                         float dt) {
    const int64_t n = c.num_voxels();
    const float sdt = dt * (1.0f / c.dx);
    auto aligned8 = [](const void* q) { return ((uintptr_t)q & 7u) == 0; };
    if (n > 0 && c.topo.num_leaves < (int64_t(1) << 22) && ns <= 1) {
        // Velocity and at most one scalar: the shared-memory leaf tile, filled from the arrays.
        advect_tile_kernel<<<(unsigned)c.topo.num_leaves, kTileThreads, 0, c.stream>>>(
            c.topo.view, static_cast<const __nv_bfloat16*>(vel), ns > 0 ? static_cast<const __half*>(sin[0]) : nullptr,
            static_cast<__nv_bfloat16*>(vel_out), ns > 0 ? static_cast<__half*>(sout[0]) : nullptr, sdt);
        HNS_LAUNCHED();
        return;
    }
    if (n > 0 && c.topo.num_leaves < (int64_t(1) << 22) && aligned8(vel) && (ns == 0 || aligned8(sin[0])) &&
        ns <= kMaxAdvectFields) {
        // Voxel records: velocity and the first scalar interleaved, then one load per tap.
        auto* rec = reinterpret_cast<uint4*>(c.scratch_f32("advect_records", (size_t)n * 2));
        pack_records_kernel<<<stream_blocks(c, n), kThreads, 0, c.stream>>>(
            static_cast<const __nv_bfloat16*>(vel), ns > 0 ? static_cast<const __half*>(sin[0]) : nullptr, rec, n);
        HNS_LAUNCHED();
        FieldSetT<__half> f{};
        f.count = std::max(0, ns - 1);
        for (int q = 0; q < f.count; ++q) {
            f.in[q] = static_cast<const __half*>(sin[1 + q]);
            f.out[q] = static_cast<__half*>(sout[1 + q]);
        }
        advect_records_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, reinterpret_cast<const uint2*>(rec), static_cast<__nv_bfloat16*>(vel_out),
            ns > 0 ? static_cast<__half*>(sout[0]) : nullptr, f, sdt);
        HNS_LAUNCHED();
        return;
    }
    int base = 0;
    do {
        FieldSetT<__half> f{};
        f.count = std::min(kMaxAdvectFields, ns - base);
        for (int q = 0; q < f.count; ++q) {
            f.in[q] = static_cast<const __half*>(sin[base + q]);
            f.out[q] = static_cast<__half*>(sout[base + q]);
        }
        const auto* vi = static_cast<const __nv_bfloat16*>(vel);
        auto* vo = base == 0 ? static_cast<__nv_bfloat16*>(vel_out) : nullptr;
        if (c.topo.num_leaves < (int64_t(1) << 22))
            advect_mixed_kernel<__nv_bfloat16, __half, int32_t>
                <<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vi, vo, f, sdt);
        else
            advect_mixed_kernel<__nv_bfloat16, __half, int64_t>
                <<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vi, vo, f, sdt);
        HNS_LAUNCHED();
        base += f.count;
    } while (base < ns);
}

void launch_divergence_mixed(const Context& c, const void* vel, float* div) {
    if (c.topo.num_leaves == 0) return;
    const auto* v = static_cast<const __nv_bfloat16*>(vel);
    if (((uintptr_t)vel & 1u) != 0) fail(HNS_ERR_INVALID_ARG, "BF16 velocity must be 2-byte aligned");
    if (((uintptr_t)vel & 7u) == 0)
        divergence_mixed_kernel<__nv_bfloat16, true><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, v, div, 1.0f / c.dx);
    else
        divergence_mixed_kernel<__nv_bfloat16, false><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, v, div, 1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_gradient_mixed(const Context& c, void* vel, const double* p) {
    if (c.topo.num_leaves == 0) return;
    auto* v = static_cast<__nv_bfloat16*>(vel);
    if (((uintptr_t)vel & 1u) != 0) fail(HNS_ERR_INVALID_ARG, "BF16 velocity must be 2-byte aligned");
    if (((uintptr_t)vel & 7u) == 0)
        gradient_mixed_kernel<__nv_bfloat16, true><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, v, p, 1.0f / c.dx);
    else
        gradient_mixed_kernel<__nv_bfloat16, false><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, v, p, 1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_gradient_f64(const Context& c, float* vel, const double* p) {
    if (c.topo.num_leaves == 0) return;
    if (((uintptr_t)vel & 3u) != 0) fail(HNS_ERR_INVALID_ARG, "FP32 velocity must be 4-byte aligned");
    if (((uintptr_t)vel & 15u) == 0)
        gradient_mixed_kernel<float, true><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, p, 1.0f / c.dx);
    else
        gradient_mixed_kernel<float, false><<<row_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, p, 1.0f / c.dx);
    HNS_LAUNCHED();
}

}  // namespace hns

using namespace hns;

namespace {

void check_mixed_desc(const hns_mixed_desc* d) {
    if (!d) fail(HNS_ERR_INVALID_ARG, "null step description");
    if (d->max_outer <= 0 || d->max_outer > 1000) fail(HNS_ERR_INVALID_ARG, "max_outer must be in [1, 1000]");
    if (d->inner_iterations <= 0) fail(HNS_ERR_INVALID_ARG, "inner_iterations must be positive");
    if (!(d->tolerance > 0.0) || !std::isfinite(d->tolerance)) fail(HNS_ERR_INVALID_ARG, "tolerance must be positive");
    if (!std::isfinite(d->dt)) fail(HNS_ERR_INVALID_ARG, "bad dt");
}

hns_status mixed_info(Context& c, const RefinePlan& plan, const hns_mixed_desc& d, hns_solve_info* info) {
    if (!info) return HNS_OK;
    int outer = 0;
    double res = 0.0;
    refine_result(c, plan, &outer, &res);
    info->iterations = outer * plan.inner;
    info->residual = res;
    info->initial_residual = 1.0;
    if (res > d.tolerance)
        return record_error(HNS_ERR_NOT_CONVERGED, "refined solve stopped after " + std::to_string(outer) +
                                                       " outer iterations with residual " + std::to_string(res));
    return HNS_OK;
}

// The mixed step on device arrays: advection (velocity and the ns scalars), divergence, the
// refined solve, the gradient.
RefinePlan mixed_step_device(Context& c, const void* vel_in, void* vel_out, const void* const* sin, void* const* sout, int ns,
                             const hns_mixed_desc& d) {
    const size_t n = (size_t)c.num_voxels();
    c.phase_begin(HNS_PHASE_ADVECT);
    launch_advect_mixed(c, vel_in, vel_out, sin, sout, ns, d.dt);
    c.phase_end();
    float* div = c.scratch_f32("project_div", n);
    double* p = reinterpret_cast<double*>(c.scratch_f32("refine_p", 2 * n));
    c.phase_begin(HNS_PHASE_DIVERGENCE);
    launch_divergence_mixed(c, vel_out, div);
    c.phase_end();
    c.phase_begin(HNS_PHASE_SOLVE);
    const float omega = d.omega > 0.f ? d.omega : 1.9f;
    RefinePlan plan = refine_solve<__half>(c, div, p, d.max_outer, d.inner_iterations, omega, d.tolerance, d.flags);
    c.phase_end();
    c.last_refine = plan;
    c.phase_begin(HNS_PHASE_GRADIENT);
    launch_gradient_mixed(c, vel_out, p);
    c.phase_end();
    return plan;
}

}  // namespace

extern "C" {

HNS_API hns_status hns_convert(hns_ctx* ctx, const void* src, int src_dtype, void* dst, int dst_dtype, int64_t count) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (count < 0) fail(HNS_ERR_INVALID_ARG, "negative count");
        if (count > 0 && (!src || !dst)) fail(HNS_ERR_INVALID_ARG, "null array");
        DeviceGuard g(c->device);
        convert_array(*c, src, src_dtype, dst, dst_dtype, count);
    });
}

HNS_API hns_status hns_step_mixed(hns_ctx* ctx, const void* vel_in, void* vel_out, const void* const* scalars_in,
                                  void* const* scalars_out, int nscalars, const hns_mixed_desc* desc, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        check_mixed_desc(desc);
        if (!vel_in || !vel_out || vel_in == vel_out) fail(HNS_ERR_INVALID_ARG, "bad velocity arrays");
        // 16-bit elements need 2-byte alignment; wider alignment only selects vector accesses.
        auto odd = [](const void* q) { return ((uintptr_t)q & 1u) != 0; };
        if (odd(vel_in) || odd(vel_out)) fail(HNS_ERR_INVALID_ARG, "BF16 velocity arrays must be 2-byte aligned");
        if (nscalars < 0 || (nscalars > 0 && (!scalars_in || !scalars_out))) fail(HNS_ERR_INVALID_ARG, "bad scalar arrays");
        for (int q = 0; q < nscalars; ++q)
            if (!scalars_in[q] || !scalars_out[q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
            else if (odd(scalars_in[q]) || odd(scalars_out[q]))
                fail(HNS_ERR_INVALID_ARG, "FP16 scalar arrays must be 2-byte aligned");
        DeviceGuard dg(c->device);
        const RefinePlan plan = mixed_step_device(*c, vel_in, vel_out, scalars_in, scalars_out, nscalars, *desc);
        st = mixed_info(*c, plan, *desc, info);
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_step_mixed_host(hns_ctx* ctx, float* vel, float* const* scalars, int nscalars,
                                       const hns_mixed_desc* desc, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        check_mixed_desc(desc);
        if (!vel) fail(HNS_ERR_INVALID_ARG, "null velocity");
        if (nscalars < 0 || (nscalars > 0 && !scalars)) fail(HNS_ERR_INVALID_ARG, "bad scalar arrays");
        DeviceGuard dg(c->device);
        const size_t n = (size_t)c->num_voxels();
        // Host data is FP32 (the reference's GridIndexedData); it is staged in FP32, converted
        // to BF16/FP16 on the device, stepped, and converted back. The host link is the bound:
        // only the velocity's upload and download are on the critical path. The scalars are
        // uploaded, advected along the incoming velocity, converted and downloaded on the
        // auxiliary stream while the main stream projects the velocity (the same kernels and
        // values as the device form, which advects them together with the velocity).
        for (int q = 0; q < nscalars; ++q)
            if (!scalars[q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
        float* stage = c->scratch_f32("mixed_host_stage", 3 * n);
        void* v_in = c->scratch_f32("mixed_vel_in", (3 * n + 1) / 2);
        void* v_out = c->scratch_f32("mixed_vel_out", (3 * n + 1) / 2);
        std::vector<const void*> sin((size_t)nscalars);
        std::vector<void*> sout((size_t)nscalars);
        for (int q = 0; q < nscalars; ++q) {
            sin[q] = c->scratch_f32("mixed_scalar_in_" + std::to_string(q), (n + 1) / 2);
            sout[q] = c->scratch_f32("mixed_scalar_out_" + std::to_string(q), (n + 1) / 2);
        }
        float* stage_aux = nscalars > 0 ? c->scratch_f32("mixed_host_stage_aux", n) : nullptr;
        if (nscalars > 0) c->ensure_aux();
        HNS_CUDA(cudaMemcpyAsync(stage, vel, 3 * n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        convert_array(*c, stage, HNS_DTYPE_F32, v_in, HNS_DTYPE_BF16, (int64_t)(3 * n));
        if (nscalars > 0) {
            HNS_CUDA(cudaEventRecord(c->aux_ready, c->stream));  // v_in is converted
            HNS_CUDA(cudaStreamWaitEvent(c->aux_stream, c->aux_ready, 0));
            // The launches below go to the auxiliary stream; the main one is restored on exit.
            struct StreamSwap {
                Context& ctx;
                cudaStream_t saved;
                ~StreamSwap() { ctx.stream = saved; }
            } swap{*c, c->stream};
            c->stream = c->aux_stream;
            for (int q = 0; q < nscalars; ++q) {
                HNS_CUDA(cudaMemcpyAsync(stage_aux, scalars[q], n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
                convert_array(*c, stage_aux, HNS_DTYPE_F32, const_cast<void*>(sin[q]), HNS_DTYPE_F16, (int64_t)n);
            }
            launch_advect_mixed(*c, v_in, nullptr, sin.data(), sout.data(), nscalars, desc->dt);
            for (int q = 0; q < nscalars; ++q) {
                convert_array(*c, sout[q], HNS_DTYPE_F16, stage_aux, HNS_DTYPE_F32, (int64_t)n);
                HNS_CUDA(cudaMemcpyAsync(scalars[q], stage_aux, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
            }
        }
        const RefinePlan plan = mixed_step_device(*c, v_in, v_out, nullptr, nullptr, 0, *desc);
        convert_array(*c, v_out, HNS_DTYPE_BF16, stage, HNS_DTYPE_F32, (int64_t)(3 * n));
        HNS_CUDA(cudaMemcpyAsync(vel, stage, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        if (nscalars > 0) HNS_CUDA(cudaStreamSynchronize(c->aux_stream));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        st = mixed_info(*c, plan, *desc, info);
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_last_refine(hns_ctx* ctx, hns_solve_info* info) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!info) fail(HNS_ERR_INVALID_ARG, "null info");
        if (c->last_refine.max_outer <= 0) fail(HNS_ERR_NOT_FOUND, "no refined solve has run on this context");
        DeviceGuard dg(c->device);
        int outer = 0;
        double res = 0.0;
        refine_result(*c, c->last_refine, &outer, &res);
        info->iterations = outer * c->last_refine.inner;
        info->residual = res;
        info->initial_residual = 1.0;
    });
}

HNS_API hns_status hns_refine_pressure(hns_ctx* ctx, double* p_out, int* outer_iterations, double* residual) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!p_out) fail(HNS_ERR_INVALID_ARG, "null output");
        DeviceGuard dg(c->device);
        const size_t n = (size_t)c->num_voxels();
        auto it = c->scratch.find("refine_p");
        if (it == c->scratch.end()) fail(HNS_ERR_NOT_FOUND, "no refined solve has run on this context");
        HNS_CUDA(cudaMemcpyAsync(p_out, it->second.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        int outer = 0;
        double res = 0.0;
        refine_result(*c, c->last_refine, &outer, &res);
        if (outer_iterations) *outer_iterations = outer;
        if (residual) *residual = res;
    });
}

}  // extern "C"
