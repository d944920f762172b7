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

// Block-wide FP64 sum of two values into acc[0], acc[1] (256 threads).
__device__ __forceinline__ void block_sum2(double a, double b, double* acc) {
    __shared__ double red[2][kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = a, red[1][threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        a = threadIdx.x < kThreads / 32 ? red[0][threadIdx.x] : 0.0;
        b = threadIdx.x < kThreads / 32 ? red[1][threadIdx.x] : 0.0;
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

template <typename V>
__device__ __forceinline__ float3 tap3(const V* d, int64_t s) {
    return s < 0 ? make_float3(0.f, 0.f, 0.f) : vload(d, s);
}
template <typename S>
__device__ __forceinline__ float tap1(const S* d, int64_t s) {
    return s < 0 ? 0.f : sload(d, s);
}

template <typename V>
__device__ __forceinline__ float3 tri3(const Taps& T, const V* d) {
    float x[8], y[8], z[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float3 a = tap3(d, T.s[q]);
        x[q] = a.x, y[q] = a.y, z[q] = a.z;
    }
    return make_float3(tri_lerp(T, x), tri_lerp(T, y), tri_lerp(T, z));
}

template <typename S>
__device__ __forceinline__ float tri1(const Taps& T, const S* d) {
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
template <typename V, typename S>
__global__ void __launch_bounds__(kThreads, 3) advect_mixed_kernel(TopoView t, const V* __restrict__ vel,
                                                                 V* __restrict__ vel_out, FieldSetT<S> f, float sdt) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 vo = vload(vel, s);
    const float bx = (float)i - vo.x * sdt, by = (float)j - vo.y * sdt, bz = (float)k - vo.z * sdt;
    Taps tb, tf;
    taps_at(tb, t, L, bx, by, bz);
    const float3 vf = tri3(tb, vel);
    taps_at(tf, t, L, bx + vf.x * sdt, by + vf.y * sdt, bz + vf.z * sdt);
    int64_t ns[6];
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
        vstore(vel_out, s, corr);
    }
    for (int c = 0; c < f.count; ++c) {
        const S* __restrict__ d = f.in[c];
        const float po = sload(d, s);
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
        sstore(f.out[c], s, fmaxf(mn, fminf(corr, mx)));
    }
}

// Divergence (divergence, src/Cuda/Kernel.cu:432-453) of a reduced-precision velocity into
// FP32, with sum (div dx^2)^2 accumulated in FP64 when `acc` is set.
template <typename V>
__global__ void __launch_bounds__(kThreads) divergence_mixed_kernel(TopoView t, const V* __restrict__ vel,
                                                                     float* __restrict__ div, float inv_dx, double h2) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 c = vload(vel, s);
    const float xp = (c.x + tap3(vel, slot_of(t, L, i + 1, j, k)).x) * 0.5f;
    const float xm = (c.x + tap3(vel, slot_of(t, L, i - 1, j, k)).x) * 0.5f;
    const float yp = (c.y + tap3(vel, slot_of(t, L, i, j + 1, k)).y) * 0.5f;
    const float ym = (c.y + tap3(vel, slot_of(t, L, i, j - 1, k)).y) * 0.5f;
    const float zp = (c.z + tap3(vel, slot_of(t, L, i, j, k + 1)).z) * 0.5f;
    const float zm = (c.z + tap3(vel, slot_of(t, L, i, j, k - 1)).z) * 0.5f;
    div[s] = (xp - xm + yp - ym + zp - zm) * inv_dx;
}

// u -= grad p with p in FP64 (0 outside the domain), velocity in reduced precision, in place.
template <typename V>
__global__ void __launch_bounds__(kThreads) gradient_mixed_kernel(TopoView t, V* __restrict__ vel,
                                                                   const double* __restrict__ p, float inv_dx) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    auto P = [&](int a, int b, int c) {
        const int64_t q = slot_of(t, L, a, b, c);
        return q < 0 ? 0.0 : __ldg(p + q);
    };
    const double h = 0.5 * (double)inv_dx;
    const float gx = (float)((P(i + 1, j, k) - P(i - 1, j, k)) * h);
    const float gy = (float)((P(i, j + 1, k) - P(i, j - 1, k)) * h);
    const float gz = (float)((P(i, j, k + 1) - P(i, j, k - 1)) * h);
    const float3 u = vload(vel, s);
    vstore(vel, s, make_float3(u.x - gx, u.y - gy, u.z - gz));
}

// ---- refinement --------------------------------------------------------------------------

// r = b - L p (FP64 arithmetic, r stored FP32) with b = div dx^2 and p = 0 outside the domain,
// plus sum r^2 and sum b^2 into acc. p null: p = 0 (r = b), and p_zero_out, when set, is
// cleared. One thread per half z-row of a leaf (z = 4h .. 4h + 3; 128 threads per leaf,
// kResidualLeaves leaves per CTA): its four values and those of the four x/y neighbour rows
// (the neighbour leaf's row across a face, 0 for a missing leaf) as 16-byte loads, and the two
// z neighbours past its ends (the other half of the row, or the leaf across the z face), with
// the Laplacian summed in the order +x, -x, +y, -y, +z, -z, -6 p. Half rows keep the kernel
// under 64 registers, twice the resident warps of whole rows.
constexpr int kResidualLeaves = kThreads / 128;

__device__ __forceinline__ void ld_half4(const double* __restrict__ q, double v[4]) {
    const double2 x0 = __ldg(reinterpret_cast<const double2*>(q));
    const double2 x1 = __ldg(reinterpret_cast<const double2*>(q) + 1);
    v[0] = x0.x, v[1] = x0.y, v[2] = x1.x, v[3] = x1.y;
}

__global__ void __launch_bounds__(kThreads) refine_residual_kernel(TopoView t, const float* __restrict__ div,
                                                                    const double* __restrict__ p,
                                                                    double* __restrict__ p_zero_out,
                                                                    float* __restrict__ r, double h2,
                                                                    const double* __restrict__ check, double tol2,
                                                                    double* __restrict__ acc) {
    if (converged(check, tol2)) return;
    const int64_t leaf = (int64_t)blockIdx.x * kResidualLeaves + (threadIdx.x >> 7);
    const int row = (threadIdx.x >> 1) & 63, h = threadIdx.x & 1, a = row >> 3, b = row & 7;
    double r2 = 0.0, b2 = 0.0;
    if (leaf < t.num_leaves) {
        const int64_t own = (leaf << 9) + 8 * row + 4 * h;
        const float4 d = __ldg(reinterpret_cast<const float4*>(div + own));
        const float dv[4] = {d.x, d.y, d.z, d.w};
        double res[4];
        if (p != nullptr) {
            const int* nb = t.nbr27 + leaf * 27;
            // nbr27: (dx+1)*9 + (dy+1)*3 + (dz+1); entry 13 is the leaf itself. The z face this
            // half row touches: -z for h = 0, +z for h = 1.
            const int nx = __ldg(nb + (a == 7 ? 22 : a == 0 ? 4 : 13)), ny = __ldg(nb + (b == 7 ? 16 : b == 0 ? 10 : 13));
            const int nz = __ldg(nb + (h ? 14 : 12));
            auto across = [&](int n, int rw) -> int64_t { return n < 0 ? own : ((int64_t)n << 9) + 8 * rw + 4 * h; };
            double c[4], xp[4], xm[4], yp[4], ym[4];
            ld_half4(p + own, c);
            ld_half4(p + (a < 7 ? own + 64 : across(nx, b)), xp);
            ld_half4(p + (a > 0 ? own - 64 : across(nx, 56 + b)), xm);
            ld_half4(p + (b < 7 ? own + 8 : across(ny, 8 * a)), yp);
            ld_half4(p + (b > 0 ? own - 8 : across(ny, 8 * a + 7)), ym);
            // The row's other half (inside the leaf) and the value across the z face.
            const double zin = __ldg(p + (h ? own - 1 : own + 4));
            const double zface = nz < 0 ? 0.0 : __ldg(p + ((int64_t)nz << 9) + 8 * row + (h ? 0 : 7));
            const double zlo = h ? zin : zface, zhi = h ? zface : zin;
            const bool zxp = a == 7 && nx < 0, zxm = a == 0 && nx < 0, zyp = b == 7 && ny < 0, zym = b == 0 && ny < 0;
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                const double lap = (zxp ? 0.0 : xp[z]) + (zxm ? 0.0 : xm[z]) + (zyp ? 0.0 : yp[z]) +
                                   (zym ? 0.0 : ym[z]) + (z < 3 ? c[z + 1] : zhi) + (z > 0 ? c[z - 1] : zlo) -
                                   6.0 * c[z];
                res[z] = (double)dv[z] * h2 - lap;
            }
        } else {
#pragma unroll
            for (int z = 0; z < 4; ++z) res[z] = (double)dv[z] * h2;
            if (p_zero_out != nullptr) {
                double2* pz = reinterpret_cast<double2*>(p_zero_out + own);
                pz[0] = make_double2(0.0, 0.0);
                pz[1] = make_double2(0.0, 0.0);
            }
        }
        *reinterpret_cast<float4*>(r + own) = make_float4((float)res[0], (float)res[1], (float)res[2], (float)res[3]);
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

// p += s e (FP64), pointwise; e in the inner solve's layout kLayout.
template <typename TI, int kLayout>
__global__ void __launch_bounds__(kThreads) refine_update_kernel(double* __restrict__ p, const TI* __restrict__ e,
                                                                  int64_t n, const float* __restrict__ scale,
                                                                  const double* __restrict__ check, double tol2) {
    if (converged(check, tol2)) return;
    const double sc = (double)*scale;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        p[q] += sc * (double)sload(e, inner_slot<kLayout>(q));
}

unsigned residual_blocks(const Context& c) {
    return (unsigned)((c.topo.num_leaves + kResidualLeaves - 1) / kResidualLeaves);
}

unsigned stream_blocks(const Context& c, int64_t n) {
    const int64_t b = (n + kThreads * 4 - 1) / (kThreads * 4);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
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
    // The FP16 inner solve's layout is an option (colour-split, colour-packed or plain order).
    const int layout = sizeof(TI) == 2 ? c.inner_layout : HNS_INNER_ROWS;
    const bool packed = layout == HNS_INNER_PACKED;
    // Colour-split: e in place with one extra all-zero leaf, and the face-neighbour table.
    TI* e_split = nullptr;
    int* nb8 = nullptr;
    if (layout == HNS_INNER_SPLIT) {
        e_split = reinterpret_cast<TI*>(c.scratch_f32("refine_e_split", ((size_t)(n + 512) * sizeof(TI) + 3) / 4));
        nb8 = reinterpret_cast<int*>(c.scratch_f32("refine_split_nb8", (size_t)c.topo.num_leaves * 8));
        HNS_CUDA(cudaMemsetAsync(e_split + n, 0, 512 * sizeof(TI), c.stream));
        launch_split_face_table(c, nb8);
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
    refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, div, nullptr, p, r, h2,
                                                                                   nullptr, tol2, plan.slots);
    HNS_LAUNCHED();
    for (int k = 0; k < plan.max_outer; ++k) {
        const double* chk = plan.slots + 2 * k;
        if (flags & HNS_SOLVE_MULTIGRID) {
            // One V-cycle on the scaled residual in FP32 (slot order), then p += s e.
            float* rm = c.scratch_f32("mg_rhat", (size_t)n);
            float* em = c.scratch_f32("mg_e", (size_t)n);
            refine_scale_kernel<float, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(r, rm, n, chk, tol2, scales + k);
            HNS_LAUNCHED();
            c.phase_begin(HNS_PHASE_INNER);
            mg_vcycle(c, rm, em, chk, tol2);
            c.phase_end();
            refine_update_kernel<float, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(p, em, n, scales + k, chk, tol2);
            HNS_LAUNCHED();
            refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, div, p, nullptr, r, h2, chk, tol2, plan.slots + 2 * (k + 1));
            HNS_LAUNCHED();
            continue;
        }
        if (layout == HNS_INNER_PACKED)
            refine_scale_kernel<TI, HNS_INNER_PACKED><<<g, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        else if (layout == HNS_INNER_SPLIT)
            refine_scale_kernel<TI, HNS_INNER_SPLIT><<<g, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        else
            refine_scale_kernel<TI, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(r, rhat, n, chk, tol2, scales + k);
        HNS_LAUNCHED();
        if (packed) launch_rhs_halo_pack(c, rhat, halo, chk, tol2);
        const TI* src = nullptr;
        const void* src_faces = nullptr;
        c.phase_begin(HNS_PHASE_INNER);
        for (int it = 0; it < plan.inner; ++it) {
            TI* dst = e[it & 1];
            if constexpr (sizeof(TI) == 2) {
                if (layout == HNS_INNER_SPLIT) {
                    // In place: red, then black.
                    dst = e_split;
                    launch_rbgs_split_half(c, nb8, rhat, dst, 0, it == 0, omega, chk, tol2);
                    launch_rbgs_split_half(c, nb8, rhat, dst, 1, false, omega, chk, tol2);
                } else if (packed) {
                    launch_rbgs_packed_half(c, rhat, halo, src, src_faces, dst, faces[it & 1], omega, chk, tol2);
                    src_faces = faces[it & 1];
                } else
                    launch_rbgs_bulk_half(c, rhat, src, dst, omega, chk, tol2);
            } else
                launch_rbgs_bulk_unit(c, reinterpret_cast<const float*>(rhat), reinterpret_cast<const float*>(src),
                                      reinterpret_cast<float*>(dst), omega, chk, tol2);
            src = dst;
        }
        c.phase_end();
        if (layout == HNS_INNER_PACKED)
            refine_update_kernel<TI, HNS_INNER_PACKED><<<g, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2);
        else if (layout == HNS_INNER_SPLIT)
            refine_update_kernel<TI, HNS_INNER_SPLIT><<<g, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2);
        else
            refine_update_kernel<TI, HNS_INNER_ROWS><<<g, kThreads, 0, c.stream>>>(p, src, n, scales + k, chk, tol2);
        HNS_LAUNCHED();
        refine_residual_kernel<<<residual_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, div, p, nullptr, r, h2, chk, tol2, plan.slots + 2 * (k + 1));
        HNS_LAUNCHED();
    }
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

void launch_advect_mixed(const Context& c, const void* vel, void* vel_out, const void* const* sin, void* const* sout, int ns,
                         float dt) {
    int base = 0;
    do {
        FieldSetT<__half> f{};
        f.count = std::min(kMaxAdvectFields, ns - base);
        for (int q = 0; q < f.count; ++q) {
            f.in[q] = static_cast<const __half*>(sin[base + q]);
            f.out[q] = static_cast<__half*>(sout[base + q]);
        }
        advect_mixed_kernel<__nv_bfloat16, __half><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, static_cast<const __nv_bfloat16*>(vel), base == 0 ? static_cast<__nv_bfloat16*>(vel_out) : nullptr, f,
            dt * (1.0f / c.dx));
        HNS_LAUNCHED();
        base += f.count;
    } while (base < ns);
}

void launch_divergence_mixed(const Context& c, const void* vel, float* div) {
    divergence_mixed_kernel<__nv_bfloat16><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
        c.topo.view, static_cast<const __nv_bfloat16*>(vel), div, 1.0f / c.dx, (double)c.dx * (double)c.dx);
    HNS_LAUNCHED();
}

void launch_gradient_mixed(const Context& c, void* vel, const double* p) {
    gradient_mixed_kernel<__nv_bfloat16><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view,
                                                                                     static_cast<__nv_bfloat16*>(vel), p,
                                                                                     1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_gradient_f64(const Context& c, float* vel, const double* p) {
    gradient_mixed_kernel<float><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, p, 1.0f / c.dx);
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

// after_advect, when given, runs on the host once the advection is enqueued (the scalars'
// outputs are final from then on; the velocity is not).
RefinePlan mixed_step_device(Context& c, const void* vel_in, void* vel_out, const void* const* sin, void* const* sout, int ns,
                             const hns_mixed_desc& d, const std::function<void()>& after_advect = {}) {
    const size_t n = (size_t)c.num_voxels();
    c.phase_begin(HNS_PHASE_ADVECT);
    launch_advect_mixed(c, vel_in, vel_out, sin, sout, ns, d.dt);
    c.phase_end();
    if (after_advect) after_advect();
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
        if (nscalars < 0 || (nscalars > 0 && (!scalars_in || !scalars_out))) fail(HNS_ERR_INVALID_ARG, "bad scalar arrays");
        for (int q = 0; q < nscalars; ++q)
            if (!scalars_in[q] || !scalars_out[q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
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
        // to BF16/FP16 on the device, stepped, and converted back.
        float* stage = c->scratch_f32("mixed_host_stage", 3 * n);
        void* v_in = c->scratch_f32("mixed_vel_in", (3 * n + 1) / 2);
        void* v_out = c->scratch_f32("mixed_vel_out", (3 * n + 1) / 2);
        std::vector<const void*> sin((size_t)nscalars);
        std::vector<void*> sout((size_t)nscalars);
        HNS_CUDA(cudaMemcpyAsync(stage, vel, 3 * n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        convert_array(*c, stage, HNS_DTYPE_F32, v_in, HNS_DTYPE_BF16, (int64_t)(3 * n));
        for (int q = 0; q < nscalars; ++q) {
            if (!scalars[q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
            void* a = c->scratch_f32("mixed_scalar_in_" + std::to_string(q), (n + 1) / 2);
            sout[q] = c->scratch_f32("mixed_scalar_out_" + std::to_string(q), (n + 1) / 2);
            sin[q] = a;
            HNS_CUDA(cudaMemcpyAsync(stage, scalars[q], n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
            convert_array(*c, stage, HNS_DTYPE_F32, a, HNS_DTYPE_F16, (int64_t)n);
        }
        // The advected scalars are final before the pressure solve: they are converted and
        // downloaded on the auxiliary stream while the main stream projects the velocity.
        float* stage_aux = nscalars > 0 ? c->scratch_f32("mixed_host_stage_aux", n) : nullptr;
        if (nscalars > 0) c->ensure_aux();
        auto download_scalars = [&] {
            HNS_CUDA(cudaEventRecord(c->aux_ready, c->stream));
            HNS_CUDA(cudaStreamWaitEvent(c->aux_stream, c->aux_ready, 0));
            // The conversions below launch on the auxiliary stream; the main one is restored on exit.
            struct StreamSwap {
                Context& ctx;
                cudaStream_t saved;
                ~StreamSwap() { ctx.stream = saved; }
            } swap{*c, c->stream};
            c->stream = c->aux_stream;
            for (int q = 0; q < nscalars; ++q) {
                convert_array(*c, sout[q], HNS_DTYPE_F16, stage_aux, HNS_DTYPE_F32, (int64_t)n);
                HNS_CUDA(cudaMemcpyAsync(scalars[q], stage_aux, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
            }
        };
        const RefinePlan plan = mixed_step_device(*c, v_in, v_out, sin.data(), sout.data(), nscalars, *desc,
                                                  nscalars > 0 ? std::function<void()>(download_scalars)
                                                               : std::function<void()>());
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
