// Adjoint (reverse-mode) kernels of the step's operators: MacCormack advection of a scalar
// and of the velocity, divergence, the red-black SOR solve from p = 0, gradient subtraction and
// vorticity confinement. Each computes the transpose of the derivative of its forward operator
// (hns_kernels.cu, hns_advance.cu) at the given inputs and ADDS it into the caller's adjoint
// arrays, so adjoints of several uses of one field accumulate.
//
// The derivatives are those of the forward arithmetic with exact real operations: the
// positions of a trace and the floor() of a trilinear sample are recomputed exactly as the
// forward computes them, and the MacCormack clamp routes the adjoint to the value it selected
// (the corrected value, or the minimum or maximum of the clamp set). Scatters (the transposes
// of trilinear samples and of the curl) use FP32 atomics; everything else is a gather.
#include <cuda_runtime.h>

#include <cmath>

#include "hns_internal.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

constexpr int kThreads = 256;

unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void coords_of(const TopoView& t, int64_t s, int& i, int& j, int& k) {
    const int4 o = t.origin[s >> 9];
    const int n = (int)(s & 511);
    i = o.x + ((n >> 6) & 7);
    j = o.y + ((n >> 3) & 7);
    k = o.z + (n & 7);
}

// Slot of the voxel at (i, j, k), -1 outside the domain (the dense leaf table).
__device__ __forceinline__ int64_t slot_at(const TopoView& t, int i, int j, int k) {
    const int li = (i >> 3) - t.lo_x, lj = (j >> 3) - t.lo_y, lk = (k >> 3) - t.lo_z;
    if (li < 0 || lj < 0 || lk < 0 || li >= t.dim_x || lj >= t.dim_y || lk >= t.dim_z) return -1;
    const int l = t.lookup[((int64_t)li * t.dim_y + lj) * t.dim_z + lk];
    return l < 0 ? -1 : ((int64_t)l << 9) + (((i & 7) << 6) | ((j & 7) << 3) | (k & 7));
}

__device__ __forceinline__ float val_s(const float* d, int64_t s) { return s < 0 ? 0.f : __ldg(d + s); }

// The forward's trilinear samples (hns_stencil.cuh tri_s / tri_v: floor, fractions, lerp along
// z, then y, then x, 0 outside), with the dense leaf table for the taps: the adjoint recomputes
// the trace exactly as the forward computed it.
__device__ __forceinline__ float ftri_s(const TopoView& t, const float* d, float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
    const float v000 = val_s(d, slot_at(t, i, j, k)), v001 = val_s(d, slot_at(t, i, j, k + 1));
    const float v010 = val_s(d, slot_at(t, i, j + 1, k)), v011 = val_s(d, slot_at(t, i, j + 1, k + 1));
    const float v100 = val_s(d, slot_at(t, i + 1, j, k)), v101 = val_s(d, slot_at(t, i + 1, j, k + 1));
    const float v110 = val_s(d, slot_at(t, i + 1, j + 1, k)), v111 = val_s(d, slot_at(t, i + 1, j + 1, k + 1));
    const float z0 = dev::lerp1(v000, v001, tz), z1 = dev::lerp1(v010, v011, tz);
    const float z2 = dev::lerp1(v100, v101, tz), z3 = dev::lerp1(v110, v111, tz);
    return dev::lerp1(dev::lerp1(z0, z1, ty), dev::lerp1(z2, z3, ty), tx);
}

__device__ __forceinline__ float3 ftri_v(const TopoView& t, const float* d, float x, float y, float z) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
    float r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        auto v = [&](int a, int b, int cc) {
            const int64_t q = slot_at(t, i + a, j + b, k + cc);
            return q < 0 ? 0.f : __ldg(d + 3 * q + c);
        };
        const float z0 = dev::lerp1(v(0, 0, 0), v(0, 0, 1), tz), z1 = dev::lerp1(v(0, 1, 0), v(0, 1, 1), tz);
        const float z2 = dev::lerp1(v(1, 0, 0), v(1, 0, 1), tz), z3 = dev::lerp1(v(1, 1, 0), v(1, 1, 1), tz);
        r[c] = dev::lerp1(dev::lerp1(z0, z1, ty), dev::lerp1(z2, z3, ty), tx);
    }
    return make_float3(r[0], r[1], r[2]);
}

// A trilinear sample's taps (slot, -1 outside), weights and the weights' derivatives with
// respect to the sample position, for the cell floor(x), floor(y), floor(z) (the forward's
// TrilinearSampler: weights (1-t) / t per axis).
struct Tri {
    int64_t s[8];
    float w[8];
    float gx[8], gy[8], gz[8];
};

__device__ __forceinline__ void tri_taps(const TopoView& t, float x, float y, float z, Tri& T) {
    const int i = __float2int_rd(x), j = __float2int_rd(y), k = __float2int_rd(z);
    const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int a = q >> 2, b = (q >> 1) & 1, c = q & 1;
        const float wx = a ? tx : 1.f - tx, wy = b ? ty : 1.f - ty, wz = c ? tz : 1.f - tz;
        const float sx = a ? 1.f : -1.f, sy = b ? 1.f : -1.f, sz = c ? 1.f : -1.f;
        T.s[q] = slot_at(t, i + a, j + b, k + c);
        T.w[q] = wx * wy * wz;
        T.gx[q] = sx * wy * wz;
        T.gy[q] = wx * sy * wz;
        T.gz[q] = wx * wy * sz;
    }
}

// Value and position gradient of a trilinear sample of scalar field d (0 outside).
__device__ __forceinline__ float tri_grad(const Tri& T, const float* d, float3& g) {
    float v = 0.f;
    g = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float f = val_s(d, T.s[q]);
        v += T.w[q] * f;
        g.x += T.gx[q] * f;
        g.y += T.gy[q] * f;
        g.z += T.gz[q] * f;
    }
    return v;
}

// The same for component c of a vec3 field.
__device__ __forceinline__ void tri_grad_c(const Tri& T, const float* vel, int c, float3& g) {
    g = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float f = T.s[q] < 0 ? 0.f : __ldg(vel + 3 * T.s[q] + c);
        g.x += T.gx[q] * f;
        g.y += T.gy[q] * f;
        g.z += T.gz[q] * f;
    }
}

__device__ __forceinline__ void scatter_s(const Tri& T, float* bar, float a) {
    if (a == 0.f) return;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (T.s[q] >= 0) atomicAdd(bar + T.s[q], a * T.w[q]);
}

__device__ __forceinline__ void scatter_v(const Tri& T, float* bar, float3 a) {
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (T.s[q] >= 0) {
            atomicAdd(bar + 3 * T.s[q], a.x * T.w[q]);
            atomicAdd(bar + 3 * T.s[q] + 1, a.y * T.w[q]);
            atomicAdd(bar + 3 * T.s[q] + 2, a.z * T.w[q]);
        }
}

__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// The clamp of MacCormack (advect_scalar / advect_vector): out = max(mn, min(corr, mx)) with
// mn/mx over {centre, 6 face neighbours, forward sample}. Returns which value the output is:
// -1 corr, 0 centre, 1..6 a neighbour (+x, -x, +y, -y, +z, -z), 7 the forward sample.
__device__ __forceinline__ int clamp_pick(float corr, float ctr, const float nbr[6], float fwd) {
    float mn = ctr, mx = ctr;
    int imn = 0, imx = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        if (nbr[q] < mn) mn = nbr[q], imn = q + 1;
        if (nbr[q] > mx) mx = nbr[q], imx = q + 1;
    }
    if (fwd < mn) mn = fwd, imn = 7;
    if (fwd > mx) mx = fwd, imx = 7;
    if (corr > mx) return imx;
    if (corr < mn) return imn;
    return -1;
}

__device__ __forceinline__ void face_offset(int q, int& di, int& dj, int& dk) {
    di = q == 0 ? 1 : q == 1 ? -1 : 0;
    dj = q == 2 ? 1 : q == 3 ? -1 : 0;
    dk = q == 4 ? 1 : q == 5 ? -1 : 0;
}

// ---- advection ------------------------------------------------------------------------------

// Adjoint of advect_scalar (in -> out along vel): in_bar += d out/d in ^T out_bar and
// vel_bar += d out/d vel ^T out_bar.
__global__ void __launch_bounds__(kThreads) adj_advect_scalar_kernel(TopoView t, const float* __restrict__ vel,
                                                                     const float* __restrict__ in,
                                                                     const float* __restrict__ out_bar,
                                                                     float* __restrict__ in_bar,
                                                                     float* __restrict__ vel_bar, float sdt, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    const float ob = __ldg(out_bar + s);
    if (ob == 0.f) return;
    int i, j, k;
    coords_of(t, s, i, j, k);
    const float po = __ldg(in + s);
    const float3 vc = make_float3(__ldg(vel + 3 * s), __ldg(vel + 3 * s + 1), __ldg(vel + 3 * s + 2));
    const float bx = (float)i - vc.x * sdt, by = (float)j - vc.y * sdt, bz = (float)k - vc.z * sdt;
    Tri tb, tf;
    tri_taps(t, bx, by, bz, tb);
    float3 gpf;
    (void)tri_grad(tb, in, gpf);
    // The trace and the clamp decision use the forward's own samples.
    const float3 vff = ftri_v(t, vel, bx, by, bz);
    const float pff = ftri_s(t, in, bx, by, bz);
    const float fx = bx + vff.x * sdt, fy = by + vff.y * sdt, fz = bz + vff.z * sdt;
    tri_taps(t, fx, fy, fz, tf);
    float3 gpb;
    (void)tri_grad(tf, in, gpb);
    const float pbf = ftri_s(t, in, fx, fy, fz);
    const float corr = pff + 0.5f * (po - pbf);
    float nbr[6];
    int64_t ns[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        int di, dj, dk;
        face_offset(q, di, dj, dk);
        ns[q] = slot_at(t, i + di, j + dj, k + dk);
        nbr[q] = val_s(in, ns[q]);
    }
    const int pick = clamp_pick(corr, po, nbr, pff);
    float g_po = 0.f, g_pf = 0.f, g_pb = 0.f;
    if (pick < 0) {
        g_pf = ob, g_po = 0.5f * ob, g_pb = -0.5f * ob;
    } else if (pick == 0) {
        g_po = ob;
    } else if (pick == 7) {
        g_pf = ob;
    } else if (ns[pick - 1] >= 0) {
        atomicAdd(in_bar + ns[pick - 1], ob);  // a neighbour outside the domain is the constant 0
    }
    if (g_po != 0.f) atomicAdd(in_bar + s, g_po);
    scatter_s(tb, in_bar, g_pf);
    scatter_s(tf, in_bar, g_pb);
    // Position adjoints: pf at back, pb at fwd = back + vf(back) * sdt, back = x - vc * sdt.
    float3 fb = make_float3(g_pb * gpb.x, g_pb * gpb.y, g_pb * gpb.z);
    float3 bb = make_float3(g_pf * gpf.x + fb.x, g_pf * gpf.y + fb.y, g_pf * gpf.z + fb.z);
    const float3 vfb = make_float3(fb.x * sdt, fb.y * sdt, fb.z * sdt);
    if (vfb.x != 0.f || vfb.y != 0.f || vfb.z != 0.f) {
        scatter_v(tb, vel_bar, vfb);
        float3 g;
        tri_grad_c(tb, vel, 0, g);
        bb.x += vfb.x * g.x, bb.y += vfb.x * g.y, bb.z += vfb.x * g.z;
        tri_grad_c(tb, vel, 1, g);
        bb.x += vfb.y * g.x, bb.y += vfb.y * g.y, bb.z += vfb.y * g.z;
        tri_grad_c(tb, vel, 2, g);
        bb.x += vfb.z * g.x, bb.y += vfb.z * g.y, bb.z += vfb.z * g.z;
    }
    if (bb.x != 0.f) atomicAdd(vel_bar + 3 * s, -sdt * bb.x);
    if (bb.y != 0.f) atomicAdd(vel_bar + 3 * s + 1, -sdt * bb.y);
    if (bb.z != 0.f) atomicAdd(vel_bar + 3 * s + 2, -sdt * bb.z);
}

// Adjoint of advect_vector (self-advection of vel): vel_bar += d out/d vel ^T out_bar, through
// the advected field and through the trace.
__global__ void __launch_bounds__(kThreads) adj_advect_vec3_kernel(TopoView t, const float* __restrict__ vel,
                                                                   const float* __restrict__ out_bar,
                                                                   float* __restrict__ vel_bar, float sdt, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    const float ob[3] = {__ldg(out_bar + 3 * s), __ldg(out_bar + 3 * s + 1), __ldg(out_bar + 3 * s + 2)};
    if (ob[0] == 0.f && ob[1] == 0.f && ob[2] == 0.f) return;
    int i, j, k;
    coords_of(t, s, i, j, k);
    const float vo[3] = {__ldg(vel + 3 * s), __ldg(vel + 3 * s + 1), __ldg(vel + 3 * s + 2)};
    const float bx = (float)i - vo[0] * sdt, by = (float)j - vo[1] * sdt, bz = (float)k - vo[2] * sdt;
    const float3 vf = ftri_v(t, vel, bx, by, bz);
    const float fx = bx + vf.x * sdt, fy = by + vf.y * sdt, fz = bz + vf.z * sdt;
    const float3 vb = ftri_v(t, vel, fx, fy, fz);
    Tri tb, tf;
    tri_taps(t, bx, by, bz, tb);
    tri_taps(t, fx, fy, fz, tf);
    int64_t ns[6];
    float nv[6][3];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        int di, dj, dk;
        face_offset(q, di, dj, dk);
        ns[q] = slot_at(t, i + di, j + dj, k + dk);
#pragma unroll
        for (int c = 0; c < 3; ++c) nv[q][c] = ns[q] < 0 ? 0.f : __ldg(vel + 3 * ns[q] + c);
    }
    const float vfa[3] = {vf.x, vf.y, vf.z}, vba[3] = {vb.x, vb.y, vb.z};
    float gvo[3] = {0.f, 0.f, 0.f}, gvf[3] = {0.f, 0.f, 0.f}, gvb[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float corr = vfa[c] + 0.5f * (vo[c] - vba[c]);
        float nbr[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) nbr[q] = nv[q][c];
        const int pick = clamp_pick(corr, vo[c], nbr, vfa[c]);
        if (pick < 0) {
            gvf[c] = ob[c], gvo[c] = 0.5f * ob[c], gvb[c] = -0.5f * ob[c];
        } else if (pick == 0) {
            gvo[c] = ob[c];
        } else if (pick == 7) {
            gvf[c] = ob[c];
        } else if (ob[c] != 0.f && ns[pick - 1] >= 0) {
            atomicAdd(vel_bar + 3 * ns[pick - 1] + c, ob[c]);
        }
    }
    // vb = tri(vel, fwd): field part and position part.
    scatter_v(tf, vel_bar, make_float3(gvb[0], gvb[1], gvb[2]));
    float3 fb = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (gvb[c] == 0.f) continue;
        float3 g;
        tri_grad_c(tf, vel, c, g);
        fb.x += gvb[c] * g.x, fb.y += gvb[c] * g.y, fb.z += gvb[c] * g.z;
    }
    // fwd = back + vf * sdt: vf gets fwd_bar * sdt; back gets fwd_bar.
    const float gvf_tot[3] = {gvf[0] + fb.x * sdt, gvf[1] + fb.y * sdt, gvf[2] + fb.z * sdt};
    scatter_v(tb, vel_bar, make_float3(gvf_tot[0], gvf_tot[1], gvf_tot[2]));
    float3 bb = fb;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (gvf_tot[c] == 0.f) continue;
        float3 g;
        tri_grad_c(tb, vel, c, g);
        bb.x += gvf_tot[c] * g.x, bb.y += gvf_tot[c] * g.y, bb.z += gvf_tot[c] * g.z;
    }
    // back = x - vo * sdt.
    atomicAdd(vel_bar + 3 * s, gvo[0] - sdt * bb.x);
    atomicAdd(vel_bar + 3 * s + 1, gvo[1] - sdt * bb.y);
    atomicAdd(vel_bar + 3 * s + 2, gvo[2] - sdt * bb.z);
}

// ---- projection -----------------------------------------------------------------------------

// Adjoint of divergence (a gather): vel_bar(s) += inv_dx / 2 (div_bar(s - e_d) - div_bar(s + e_d)).
__global__ void __launch_bounds__(kThreads) adj_divergence_kernel(TopoView t, const float* __restrict__ div_bar,
                                                                  float* __restrict__ vel_bar, float h, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    int i, j, k;
    coords_of(t, s, i, j, k);
    vel_bar[3 * s] += h * (val_s(div_bar, slot_at(t, i - 1, j, k)) - val_s(div_bar, slot_at(t, i + 1, j, k)));
    vel_bar[3 * s + 1] += h * (val_s(div_bar, slot_at(t, i, j - 1, k)) - val_s(div_bar, slot_at(t, i, j + 1, k)));
    vel_bar[3 * s + 2] += h * (val_s(div_bar, slot_at(t, i, j, k - 1)) - val_s(div_bar, slot_at(t, i, j, k + 1)));
}

// Adjoint of subtract_gradient (out = vel - grad p) with respect to p (a gather):
// p_bar(s) += inv_dx / 2 sum_d (out_bar_d(s + e_d) - out_bar_d(s - e_d)).
__global__ void __launch_bounds__(kThreads) adj_gradient_kernel(TopoView t, const float* __restrict__ out_bar,
                                                                float* __restrict__ p_bar, float h, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    int i, j, k;
    coords_of(t, s, i, j, k);
    auto ob = [&](int64_t q, int c) { return q < 0 ? 0.f : __ldg(out_bar + 3 * q + c); };
    const float g = (ob(slot_at(t, i + 1, j, k), 0) - ob(slot_at(t, i - 1, j, k), 0)) +
                    (ob(slot_at(t, i, j + 1, k), 1) - ob(slot_at(t, i, j - 1, k), 1)) +
                    (ob(slot_at(t, i, j, k + 1), 2) - ob(slot_at(t, i, j, k - 1), 2));
    p_bar[s] += h * g;
}

// Adjoint of one colour-c half-sweep of redBlackGaussSeidelUpdate, in place on lam. The forward
// half-sweep sets p(c) = (1 - omega) p(c) + omega / 6 (sum of the neighbours - div dx^2) on
// colour c and keeps colour c'; its transpose, from the adjoint lam' after it, gives
//   lam(c') = lam'(c') + omega / 6 sum of the (colour c) neighbours of lam',
//   div_bar(c) -= dx^2 omega / 6 lam'(c),   lam(c) = (1 - omega) lam'(c).
// The last factor is uniform over a colour, so the caller keeps it as a scale per colour: the
// true lam is scale_colour x the stored values. This launch writes colour c' fully scaled
// (keep = the old scale of c', nbr = omega / 6 x the scale of c) and only reads colour c, so it
// runs in place; the caller then sets the scale of c' to 1 and multiplies that of c by
// (1 - omega).
//
// One thread per z-row of a leaf (64 per leaf, 4 leaves per CTA): it loads its row and the four
// x/y neighbour rows as 32-byte vectors (the neighbour leaf's row across a face, zeros for a
// missing leaf) and the two values across the z faces, updates the 4 voxels of colour c' and
// stores them one by one (the row's colour-c values are read by other threads), and updates
// div_bar on the 4 voxels of colour c of its row, which only it touches.
constexpr int kRowLeavesPerBlock = 4;

__device__ __forceinline__ void ld_row(const float* __restrict__ p, float v[8]) {
    const float4 lo = *reinterpret_cast<const float4*>(p), hi = *reinterpret_cast<const float4*>(p + 4);
    v[0] = lo.x, v[1] = lo.y, v[2] = lo.z, v[3] = lo.w, v[4] = hi.x, v[5] = hi.y, v[6] = hi.z, v[7] = hi.w;
}

__global__ void __launch_bounds__(64 * kRowLeavesPerBlock) adj_rbgs_colour_kernel(TopoView t, float* lam,
                                                                                  float* __restrict__ div_bar,
                                                                                  int colour, float keep, float nbr,
                                                                                  float dmul) {
    const int64_t leaf = (int64_t)blockIdx.x * kRowLeavesPerBlock + (threadIdx.x >> 6);
    if (leaf >= t.num_leaves) return;
    const int r = threadIdx.x & 63, a = r >> 3, b = r & 7;
    const int* nb = t.nbr27 + leaf * 27;
    // nbr27: (dx+1)*9 + (dy+1)*3 + (dz+1); entry 13 is the leaf itself.
    const int nx = __ldg(nb + (a == 7 ? 22 : a == 0 ? 4 : 13)), ny = __ldg(nb + (b == 7 ? 16 : b == 0 ? 10 : 13));
    const int nzm = __ldg(nb + 12), nzp = __ldg(nb + 14);
    const int64_t own = (leaf << 9) + 8 * r;
    // Rows (a +- 1, b) and (a, b +- 1): in this leaf, or across the face (missing: this row, zeroed).
    auto across = [&](int n, int row) -> int64_t { return n < 0 ? own : ((int64_t)n << 9) + 8 * row; };
    const int64_t oxp = a < 7 ? own + 64 : across(nx, b), oxm = a > 0 ? own - 64 : across(nx, 56 + b);
    const int64_t oyp = b < 7 ? own + 8 : across(ny, 8 * a), oym = b > 0 ? own - 8 : across(ny, 8 * a + 7);
    const bool zxp = a == 7 && nx < 0, zxm = a == 0 && nx < 0, zyp = b == 7 && ny < 0, zym = b == 0 && ny < 0;
    float c[8], xp[8], xm[8], yp[8], ym[8];
    ld_row(lam + own, c);
    ld_row(lam + oxp, xp);
    ld_row(lam + oxm, xm);
    ld_row(lam + oyp, yp);
    ld_row(lam + oym, ym);
    const float zlo = nzm < 0 ? 0.f : lam[((int64_t)nzm << 9) + 8 * r + 7];
    const float zhi = nzp < 0 ? 0.f : lam[((int64_t)nzp << 9) + 8 * r];
    float d[8];
    ld_row(div_bar + own, d);
    const int pc = (a + b + colour) & 1;  // z parity of colour c in this row
#pragma unroll
    for (int z = 0; z < 8; ++z) {
        if ((z & 1) == pc) {
            d[z] -= dmul * c[z];
        } else {
            const float sx = (zxp ? 0.f : xp[z]) + (zxm ? 0.f : xm[z]);
            const float sy = (zyp ? 0.f : yp[z]) + (zym ? 0.f : ym[z]);
            const float sz = (z < 7 ? c[z + 1] : zhi) + (z > 0 ? c[z - 1] : zlo);
            lam[own + z] = keep * c[z] + nbr * (sx + sy + sz);
        }
    }
    *reinterpret_cast<float4*>(div_bar + own) = make_float4(d[0], d[1], d[2], d[3]);
    *reinterpret_cast<float4*>(div_bar + own + 4) = make_float4(d[4], d[5], d[6], d[7]);
}

// ---- vorticity confinement ------------------------------------------------------------------

__device__ __forceinline__ float3 ldv(const float* vel, int64_t q) {
    return q < 0 ? make_float3(0.f, 0.f, 0.f) : make_float3(__ldg(vel + 3 * q), __ldg(vel + 3 * q + 1), __ldg(vel + 3 * q + 2));
}

// Curl at (i, j, k) from its six face neighbours (computeVorticityMag's differences).
__device__ __forceinline__ float3 curl_at(const TopoView& t, const float* vel, int i, int j, int k, float f) {
    const float3 px = ldv(vel, slot_at(t, i + 1, j, k)), mx = ldv(vel, slot_at(t, i - 1, j, k));
    const float3 py = ldv(vel, slot_at(t, i, j + 1, k)), my = ldv(vel, slot_at(t, i, j - 1, k));
    const float3 pz = ldv(vel, slot_at(t, i, j, k + 1)), mz = ldv(vel, slot_at(t, i, j, k - 1));
    return make_float3(((py.z - my.z) - (pz.y - mz.y)) * f, ((pz.x - mz.x) - (px.z - mx.z)) * f,
                       ((px.y - mx.y) - (py.x - my.x)) * f);
}

__device__ __forceinline__ void add_v(float* bar, int64_t q, int c, float a) {
    if (q >= 0 && a != 0.f) atomicAdd(bar + 3 * q + c, a);
}

// Transpose of the curl at (i, j, k): scatters the adjoint w of the curl into vel_bar.
__device__ __forceinline__ void curl_adjoint(const TopoView& t, float* vel_bar, int i, int j, int k, float3 w, float f) {
    const int64_t px = slot_at(t, i + 1, j, k), mx = slot_at(t, i - 1, j, k);
    const int64_t py = slot_at(t, i, j + 1, k), my = slot_at(t, i, j - 1, k);
    const int64_t pz = slot_at(t, i, j, k + 1), mz = slot_at(t, i, j, k - 1);
    add_v(vel_bar, py, 2, w.x * f), add_v(vel_bar, my, 2, -w.x * f);
    add_v(vel_bar, pz, 1, -w.x * f), add_v(vel_bar, mz, 1, w.x * f);
    add_v(vel_bar, pz, 0, w.y * f), add_v(vel_bar, mz, 0, -w.y * f);
    add_v(vel_bar, px, 2, -w.y * f), add_v(vel_bar, mx, 2, w.y * f);
    add_v(vel_bar, px, 1, w.z * f), add_v(vel_bar, mx, 1, -w.z * f);
    add_v(vel_bar, py, 0, -w.z * f), add_v(vel_bar, my, 0, w.z * f);
}

// Adjoint of vorticityConfinement: out = vel + dt scale (N x omega), N = g / (|g| + 1e-5),
// g = (|omega| at +-fs along each axis) differences * inv_dx / 2, omega = curl * inv_dx / 2.
__global__ void __launch_bounds__(kThreads) adj_confinement_kernel(TopoView t, const float* __restrict__ vel,
                                                                   const float* __restrict__ out_bar,
                                                                   float* __restrict__ vel_bar, float dt, float inv_dx,
                                                                   float scale, int fs, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    const float3 ob = make_float3(__ldg(out_bar + 3 * s), __ldg(out_bar + 3 * s + 1), __ldg(out_bar + 3 * s + 2));
    atomicAdd(vel_bar + 3 * s, ob.x);
    atomicAdd(vel_bar + 3 * s + 1, ob.y);
    atomicAdd(vel_bar + 3 * s + 2, ob.z);
    // Offset 0 (|factor_scale| < 1): both |omega| samples are the same voxel, the gradient is
    // identically 0 and so is the force; the terms below would cancel only up to rounding.
    if (fs == 0 || (ob.x == 0.f && ob.y == 0.f && ob.z == 0.f)) return;
    int i, j, k;
    coords_of(t, s, i, j, k);
    const float f = 0.5f * inv_dx;
    const float3 w = curl_at(t, vel, i, j, k, f);
    // |omega| at the six offset voxels (+x, -x, +y, -y, +z, -z), which may lie outside the domain.
    float3 wv[6];
    float m[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        int di, dj, dk;
        face_offset(q, di, dj, dk);
        wv[q] = curl_at(t, vel, i + fs * di, j + fs * dj, k + fs * dk, f);
        m[q] = sqrtf(dot3(wv[q], wv[q]));
    }
    const float3 g = make_float3((m[0] - m[1]) * f, (m[2] - m[3]) * f, (m[4] - m[5]) * f);
    const float gn = sqrtf(dot3(g, g));
    const float glen = gn + 1e-5f;
    const float3 N = make_float3(g.x / glen, g.y / glen, g.z / glen);
    // f = scale (N x omega); out_bar . (dt f).
    const float3 fb = make_float3(ob.x * dt * scale, ob.y * dt * scale, ob.z * dt * scale);
    // d(N x w) = dN x w + N x dw:  N_bar = w x fb, w_bar = fb x N.
    const float3 Nb = make_float3(w.y * fb.z - w.z * fb.y, w.z * fb.x - w.x * fb.z, w.x * fb.y - w.y * fb.x);
    const float3 wb = make_float3(fb.y * N.z - fb.z * N.y, fb.z * N.x - fb.x * N.z, fb.x * N.y - fb.y * N.x);
    curl_adjoint(t, vel_bar, i, j, k, wb, f);
    // N = g / glen: g_bar = N_bar / glen - g (N_bar . g) / (glen^2 |g|).
    float3 gb = make_float3(Nb.x / glen, Nb.y / glen, Nb.z / glen);
    if (gn > 0.f) {
        const float c = dot3(Nb, g) / (glen * glen * gn);
        gb.x -= c * g.x, gb.y -= c * g.y, gb.z -= c * g.z;
    }
    const float mb[6] = {gb.x * f, -gb.x * f, gb.y * f, -gb.y * f, gb.z * f, -gb.z * f};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        if (m[q] <= 0.f || mb[q] == 0.f) continue;
        int di, dj, dk;
        face_offset(q, di, dj, dk);
        const float r = mb[q] / m[q];
        curl_adjoint(t, vel_bar, i + fs * di, j + fs * dj, k + fs * dk, make_float3(r * wv[q].x, r * wv[q].y, r * wv[q].z), f);
    }
}

__global__ void __launch_bounds__(kThreads) accumulate_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                                              int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s < n) dst[s] += __ldg(src + s);
}

}  // namespace

void launch_adj_accumulate(const Context& c, const float* src, float* dst, int64_t n) {
    if (n <= 0) return;
    accumulate_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(src, dst, n);
    HNS_LAUNCHED();
}

void launch_adj_advect_scalar(const Context& c, const float* vel, const float* in, const float* out_bar, float* in_bar,
                              float* vel_bar, float dt) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    adj_advect_scalar_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(c.topo.view, vel, in, out_bar, in_bar, vel_bar,
                                                                       dt * (1.0f / c.dx), n);
    HNS_LAUNCHED();
}

void launch_adj_advect_vec3(const Context& c, const float* vel, const float* out_bar, float* vel_bar, float dt) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    adj_advect_vec3_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(c.topo.view, vel, out_bar, vel_bar, dt * (1.0f / c.dx), n);
    HNS_LAUNCHED();
}

void launch_adj_divergence(const Context& c, const float* div_bar, float* vel_bar) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    adj_divergence_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(c.topo.view, div_bar, vel_bar, 0.5f / c.dx, n);
    HNS_LAUNCHED();
}

void launch_adj_gradient(const Context& c, const float* out_bar, float* p_bar) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    adj_gradient_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(c.topo.view, out_bar, p_bar, 0.5f / c.dx, n);
    HNS_LAUNCHED();
}

void launch_adj_rbgs_colour(const Context& c, float* lam, float* div_bar, int colour, float keep, float nbr, float dmul) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    adj_rbgs_colour_kernel<<<(unsigned)((L + kRowLeavesPerBlock - 1) / kRowLeavesPerBlock), 64 * kRowLeavesPerBlock, 0,
                             c.stream>>>(c.topo.view, lam, div_bar, colour, keep, nbr, dmul);
    HNS_LAUNCHED();
}

void launch_adj_confinement(const Context& c, const float* vel, const float* out_bar, float* vel_bar, float dt,
                            float scale, float factor_scale) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    adj_confinement_kernel<<<blocks_for(n), kThreads, 0, c.stream>>>(c.topo.view, vel, out_bar, vel_bar, dt, 1.0f / c.dx,
                                                                     scale, (int)factor_scale, n);
    HNS_LAUNCHED();
}

}  // namespace hns

// ---- C ABI -----------------------------------------------------------------------------------

namespace hns {

// The adjoint of `iterations` red-black iterations from p = 0 (the forward's
// HNS_SOLVE_ZERO_INIT): the half-sweeps' transposes in reverse order, black first, in place on
// a copy of p_bar with one scale per colour (adj_rbgs_colour_kernel). The adjoint with respect
// to the initial p is not needed (p starts at 0), so lam is never rescaled at the end.
void adj_rbgs(Context& c, const float* p_bar, float* div_bar, int iterations, float omega) {
    if (iterations <= 0) return;
    const size_t n = (size_t)c.num_voxels();
    float* lam = c.scratch_f32("adjoint_lam", n);
    HNS_CUDA(cudaMemcpyAsync(lam, p_bar, n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
    const float a = omega * dev::kInv6;
    const float dx2 = c.dx * c.dx;
    float scale[2] = {1.f, 1.f};  // red, black
    for (int it = 0; it < iterations; ++it)
        for (int colour = 1; colour >= 0; --colour) {
            const int other = colour ^ 1;
            launch_adj_rbgs_colour(c, lam, div_bar, colour, scale[other], a * scale[colour], dx2 * a * scale[colour]);
            scale[other] = 1.f;
            scale[colour] *= 1.f - omega;
        }
}

namespace {

// vel_bar (the adjoint of the projected velocity) -> the adjoint of the velocity before the
// projection: vel_bar - D^T M^T G^T vel_bar, accumulated in place.
void adj_project(Context& c, float* vel_bar, int iterations, float omega) {
    const size_t n = (size_t)c.num_voxels();
    float* p_bar = c.scratch_f32("adjoint_p_bar", n);
    float* div_bar = c.scratch_f32("adjoint_div_bar", n);
    HNS_CUDA(cudaMemsetAsync(p_bar, 0, n * sizeof(float), c.stream));
    HNS_CUDA(cudaMemsetAsync(div_bar, 0, n * sizeof(float), c.stream));
    launch_adj_gradient(c, vel_bar, p_bar);
    adj_rbgs(c, p_bar, div_bar, iterations, omega);
    launch_adj_divergence(c, div_bar, vel_bar);
}

float default_omega(const Context& c, float omega) {
    return omega > 0.f ? omega : (float)(2.0f / (1.0f + std::sin(3.14159 * (double)c.dx)));
}

void need(const void* p, const char* what) {
    if (!p) fail(HNS_ERR_INVALID_ARG, std::string("null ") + what);
}

}  // namespace
}  // namespace hns

using namespace hns;

extern "C" {

HNS_API hns_status hns_adjoint_advect_scalar(hns_ctx* ctx, const float* vel, const float* in, const float* out_bar,
                                             float* in_bar, float* vel_bar, float dt) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(vel, "velocity"), need(in, "field"), need(out_bar, "output adjoint"), need(in_bar, "field adjoint");
        need(vel_bar, "velocity adjoint");
        DeviceGuard g(c->device);
        launch_adj_advect_scalar(*c, vel, in, out_bar, in_bar, vel_bar, dt);
    });
}

HNS_API hns_status hns_adjoint_advect_vec3(hns_ctx* ctx, const float* vel, const float* out_bar, float* vel_bar, float dt) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(vel, "velocity"), need(out_bar, "output adjoint"), need(vel_bar, "velocity adjoint");
        DeviceGuard g(c->device);
        launch_adj_advect_vec3(*c, vel, out_bar, vel_bar, dt);
    });
}

HNS_API hns_status hns_adjoint_divergence(hns_ctx* ctx, const float* div_bar, float* vel_bar) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(div_bar, "divergence adjoint"), need(vel_bar, "velocity adjoint");
        DeviceGuard g(c->device);
        launch_adj_divergence(*c, div_bar, vel_bar);
    });
}

HNS_API hns_status hns_adjoint_subtract_gradient(hns_ctx* ctx, const float* out_bar, float* vel_bar, float* p_bar) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(out_bar, "output adjoint"), need(p_bar, "pressure adjoint");
        DeviceGuard g(c->device);
        if (vel_bar != nullptr) launch_adj_accumulate(*c, out_bar, vel_bar, 3 * c->num_voxels());  // d out / d vel = I
        launch_adj_gradient(*c, out_bar, p_bar);
    });
}

HNS_API hns_status hns_adjoint_rbgs(hns_ctx* ctx, const float* p_bar, float* div_bar, int iterations, float omega) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(p_bar, "pressure adjoint"), need(div_bar, "divergence adjoint");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        DeviceGuard g(c->device);
        adj_rbgs(*c, p_bar, div_bar, iterations, omega);  // hns_rbgs takes omega as given
    });
}

HNS_API hns_status hns_adjoint_project(hns_ctx* ctx, float* vel_bar, int iterations, float omega) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(vel_bar, "velocity adjoint");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        DeviceGuard g(c->device);
        adj_project(*c, vel_bar, iterations, default_omega(*c, omega));
    });
}

HNS_API hns_status hns_adjoint_vorticity_confinement(hns_ctx* ctx, const float* vel, const float* out_bar, float* vel_bar,
                                                     float dt, float scale, float factor_scale) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(vel, "velocity"), need(out_bar, "output adjoint"), need(vel_bar, "velocity adjoint");
        if (!std::isfinite(factor_scale) || std::fabs(factor_scale) > 1e6f) fail(HNS_ERR_INVALID_ARG, "factor_scale out of range");
        DeviceGuard g(c->device);
        launch_adj_confinement(*c, vel, out_bar, vel_bar, dt, scale, factor_scale);
    });
}

HNS_API hns_status hns_adjoint_step_plain(hns_ctx* ctx, const float* vel_in, const float* const* scalars_in, int nscalars,
                                          const float* vel_out_bar, const float* const* scalars_out_bar, float* vel_in_bar,
                                          float* const* scalars_in_bar, float dt, int iterations, float omega) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        need(vel_in, "velocity"), need(vel_out_bar, "output velocity adjoint"), need(vel_in_bar, "velocity adjoint");
        if (nscalars < 0) fail(HNS_ERR_INVALID_ARG, "negative scalar count");
        if (nscalars > 0) need(scalars_in, "scalars"), need(scalars_out_bar, "scalar adjoints"), need(scalars_in_bar, "scalar adjoints");
        for (int q = 0; q < nscalars; ++q)
            need(scalars_in[q], "scalar"), need(scalars_out_bar[q], "scalar adjoint"), need(scalars_in_bar[q], "scalar adjoint");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        DeviceGuard g(c->device);
        const int64_t n3 = 3 * c->num_voxels();
        // Adjoint of the advected velocity: the output adjoint through the projection.
        float* adv_bar = c->scratch_f32("adjoint_adv_bar", (size_t)n3);
        HNS_CUDA(cudaMemcpyAsync(adv_bar, vel_out_bar, (size_t)n3 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
        adj_project(*c, adv_bar, iterations, default_omega(*c, omega));
        // Velocity self-advection and the scalars' advection along the same velocity.
        launch_adj_advect_vec3(*c, vel_in, adv_bar, vel_in_bar, dt);
        for (int q = 0; q < nscalars; ++q)
            launch_adj_advect_scalar(*c, vel_in, scalars_in[q], scalars_out_bar[q], scalars_in_bar[q], vel_in_bar, dt);
    });
}

}  // extern "C"
