// Solver kernels for sm_100a: advection, divergence, red-black SOR, gradient subtraction,
// vorticity confinement, FP64 residual norms.
//
// Work decomposition: every kernel is leaf-tiled. Stencil and advection kernels run two
// 256-thread CTAs per 8^3 leaf, one thread per voxel, with the leaf's 27-leaf neighbourhood
// staged in shared memory so that neighbour taps resolve without a tree walk (the
// reference walks a NanoVDB ReadAccessor per tap, src/Utils/Stencils.hpp:59-61). The
// red-black solver runs one CTA per leaf and fuses both colours of an iteration: it stages
// the leaf with a two-voxel pressure halo and a one-voxel divergence halo, relaxes the red
// voxels of the leaf and of its one-voxel face ring, then the black voxels of the leaf, so
// that one pass reads p and div once and writes p once (ping-pong buffers).
#include <cuda_runtime.h>

#include "hns_internal.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

using namespace dev;

constexpr int kThreads = 256;

// ---- advection ------------------------------------------------------------------------------

// MacCormack advection of the SOP-facing operators, fused: advect_vector
// (src/Cuda/Kernel.cu:349-426) for the velocity and advect_scalar (src/Cuda/Kernel.cu:294-344,
// the HNanoAdvect kernel) for any number of scalars, without collision. Both kernels trace
// the same two points -- the back-trace from the voxel's own velocity and the re-trace with
// the lerp-chain trilinear velocity there -- so the trace and the 8+8 tap addresses are
// computed once and every field is sampled from them. vel_out may be null (scalars only) and
// f.count may be 0 (velocity only); each output equals the reference kernel's.
__global__ void __launch_bounds__(kThreads, 3) advect_fused_kernel(TopoView t, const float* __restrict__ vel,
                                                                    float* __restrict__ vel_out, FieldSet f, float sdt,
                                                                    const float* __restrict__ sdf, float inv_dx) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 vo = ld3(vel, s);
    float bx = (float)i - vo.x * sdt, by = (float)j - vo.y * sdt, bz = (float)k - vo.z * sdt;
    // A collider pulls trace points inside it back: the back position to the voxel, the forward
    // one to the back position (advect_vector, src/Cuda/Kernel.cu:373-383).
    if (sdf != nullptr && sdf_inside(t, L, sdf, bx, by, bz)) bx = (float)i, by = (float)j, bz = (float)k;
    Taps tb, tf;
    taps_at(tb, t, L, bx, by, bz);
    const float3 vf = tri_v(tb, vel);
    float fx = bx + vf.x * sdt, fy = by + vf.y * sdt, fz = bz + vf.z * sdt;
    if (sdf != nullptr && sdf_inside(t, L, sdf, fx, fy, fz)) fx = bx, fy = by, fz = bz;
    taps_at(tf, t, L, fx, fy, fz);
    // Face neighbours in the reference's clamp order: x-1, x+1, y-1, y+1, z-1, z+1.
    int64_t ns[6];
    face_slots(L, s, v.n, ns);
    if (vel_out != nullptr) {
        const float3 vb = tri_v(tf, vel);
        float3 corr = make_float3(vf.x + 0.5f * (vo.x - vb.x), vf.y + 0.5f * (vo.y - vb.y), vf.z + 0.5f * (vo.z - vb.z));
        float3 mn = vo, mx = vo;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float3 a = tap_v(vel, ns[q]);
            mn.x = fminf(mn.x, a.x), mn.y = fminf(mn.y, a.y), mn.z = fminf(mn.z, a.z);
            mx.x = fmaxf(mx.x, a.x), mx.y = fmaxf(mx.y, a.y), mx.z = fmaxf(mx.z, a.z);
        }
        mn.x = fminf(mn.x, vf.x), mn.y = fminf(mn.y, vf.y), mn.z = fminf(mn.z, vf.z);
        mx.x = fmaxf(mx.x, vf.x), mx.y = fmaxf(mx.y, vf.y), mx.z = fmaxf(mx.z, vf.z);
        corr.x = fmaxf(mn.x, fminf(corr.x, mx.x));
        corr.y = fmaxf(mn.y, fminf(corr.y, mx.y));
        corr.z = fmaxf(mn.z, fminf(corr.z, mx.z));
        if (sdf != nullptr) collide(t, L, sdf, s, i, j, k, inv_dx, 1.5f, corr);  // Kernel.cu:409-419
        st3(vel_out, s, corr);
    }
    for (int c = 0; c < f.count; ++c) {
        const float* __restrict__ d = f.in[c];
        const float po = __ldg(d + s);
        const float pf = tri_s(tb, d);
        const float pb = tri_s(tf, d);
        const float corr = pf + 0.5f * (po - pb);
        float mn = po, mx = po;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float a = tap_s(d, ns[q]);
            mn = fminf(mn, a);
            mx = fmaxf(mx, a);
        }
        mn = fminf(mn, pf);
        mx = fmaxf(mx, pf);
        f.out[c][s] = fmaxf(mn, fminf(corr, mx));
    }
}

// advect_scalars (src/Cuda/Kernel.cu:163-289): taps, weights and the re-traced position are
// computed once and shared by every field. sdf (or null): a collider pulls trace points
// inside it back (Kernel.cu:192-195, 245-248).
__global__ void __launch_bounds__(kThreads) advect_scalars_kernel(TopoView t, const float* __restrict__ vel, FieldSet f,
                                                                   float sdt, const float* __restrict__ sdf) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 vc = ld3(vel, s);
    float bx = (float)i - vc.x * sdt, by = (float)j - vc.y * sdt, bz = (float)k - vc.z * sdt;
    if (sdf != nullptr && sdf_inside(t, L, sdf, bx, by, bz)) bx = (float)i, by = (float)j, bz = (float)k;
    int64_t bi[8], fi[8], ni[6];
    float bw[8], fw[8];
    interp_setup(t, L, bx, by, bz, bi, bw);
    float3 vf = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float3 a = ld3(vel, bi[q]);
        vf.x = vf.x + a.x * bw[q];
        vf.y = vf.y + a.y * bw[q];
        vf.z = vf.z + a.z * bw[q];
    }
    float fx = bx + vf.x * sdt, fy = by + vf.y * sdt, fz = bz + vf.z * sdt;
    if (sdf != nullptr && sdf_inside(t, L, sdf, fx, fy, fz)) fx = bx, fy = by, fz = bz;
    interp_setup(t, L, fx, fy, fz, fi, fw);
    ni[0] = tap_slot(t, L, i - 1, j, k);
    ni[1] = tap_slot(t, L, i + 1, j, k);
    ni[2] = tap_slot(t, L, i, j - 1, k);
    ni[3] = tap_slot(t, L, i, j + 1, k);
    ni[4] = tap_slot(t, L, i, j, k - 1);
    ni[5] = tap_slot(t, L, i, j, k + 1);
    for (int c = 0; c < f.count; ++c) {
        const float* __restrict__ d = f.in[c];
        const float po = __ldg(d + s);
        float pf = 0.f, pb = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            pf = __fmaf_rn(__ldg(d + bi[q]), bw[q], pf);
            pb = __fmaf_rn(__ldg(d + fi[q]), fw[q], pb);
        }
        const float corr = __fmaf_rn(0.5f, po - pb, pf);
        float mn = po, mx = po;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float a = __ldg(d + ni[q]);
            mn = fminf(mn, a);
            mx = fmaxf(mx, a);
        }
        mn = fminf(mn, pf);
        mx = fmaxf(mx, pf);
        f.out[c][s] = fmaxf(mn, fminf(corr, mx));
    }
}

// ---- projection -----------------------------------------------------------------------------

// divergence (src/Cuda/Kernel.cu:432-453).
__global__ void __launch_bounds__(kThreads) divergence_kernel(TopoView t, const float* __restrict__ vel,
                                                               float* __restrict__ div, float inv_dx) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 c = ld3(vel, s);
    const float xp = (c.x + near_v(t, L, vel, i + 1, j, k).x) * 0.5f;
    const float xm = (c.x + near_v(t, L, vel, i - 1, j, k).x) * 0.5f;
    const float yp = (c.y + near_v(t, L, vel, i, j + 1, k).y) * 0.5f;
    const float ym = (c.y + near_v(t, L, vel, i, j - 1, k).y) * 0.5f;
    const float zp = (c.z + near_v(t, L, vel, i, j, k + 1).z) * 0.5f;
    const float zm = (c.z + near_v(t, L, vel, i, j, k - 1).z) * 0.5f;
    div[s] = (xp - xm + yp - ym + zp - zm) * inv_dx;
}

constexpr int PT = 12;  // pressure tile edge: leaf + two-voxel halo (local -2..9)
constexpr int RT = 10;  // divergence tile edge: leaf + one-voxel halo (local -1..8)

__device__ __forceinline__ int halo_depth(int a) { return a < 0 ? -a : (a > 7 ? a - 7 : 0); }
__device__ __forceinline__ int nbr_index(int a) { return a < 0 ? 0 : (a > 7 ? 2 : 1); }

// Calls f(offset into the pressure tile) for each in-domain face neighbour of staged cell
// (a, b, d), in the order x+, x-, y+, y-, z+, z- (nb: the staged 27-leaf neighbourhood).
template <typename F>
__device__ __forceinline__ void staged_neighbours(const int* nb, int a, int b, int d, F&& f) {
    auto in = [&](int x, int y, int z) { return nb[nbr_index(x) * 9 + nbr_index(y) * 3 + nbr_index(z)] >= 0; };
    if (in(a + 1, b, d)) f(PT * PT);
    if (in(a - 1, b, d)) f(-PT * PT);
    if (in(a, b + 1, d)) f(PT);
    if (in(a, b - 1, d)) f(-PT);
    if (in(a, b, d + 1)) f(1);
    if (in(a, b, d - 1)) f(-1);
}

// The Gauss-Seidel value of staged cell q (local (a, b, d)) with right-hand side bdx2 = div dx^2:
// the reference's (sum of the six neighbours, 0 outside - bdx2) / 6, or with zero-gradient walls
// (sum of the in-domain neighbours - bdx2) / their count.
template <bool kNeumann>
__device__ __forceinline__ float relax_target(const float* sp, const int* nb, int q, int a, int b, int d, float bdx2) {
    if constexpr (kNeumann) {
        float sum = 0.f;
        int cnt = 0;
        staged_neighbours(nb, a, b, d, [&](int off) {
            sum = cnt == 0 ? sp[q + off] : sum + sp[q + off];
            ++cnt;
        });
        return (sum - bdx2) / (float)cnt;
    } else {
        const float sum = sp[q + PT * PT] + sp[q - PT * PT] + sp[q + PT] + sp[q - PT] + sp[q + 1] + sp[q - 1];
        return (sum - bdx2) * kInv6;
    }
}

// One red+black iteration of redBlackGaussSeidelUpdate (src/Cuda/Kernel.cu:459-489):
// the reference's two launches per iteration (src/Cuda/HNanoSolver.cu:367-372) fused into
// one pass. Red (colour 0) voxels of the leaf and of its face ring are relaxed from the old
// black values; black voxels of the leaf then use the new red values. The ring's red values
// equal what the neighbouring CTA computes for them (same inputs, same arithmetic), so the
// result is that of the two-launch sweep. p is read from p_in (zero when null) and written
// to p_out. Cells outside the domain hold p = 0 and are never relaxed (Dirichlet-0 walls).
//
// Device-side convergence: `check` (when set) holds {sum r^2, sum b^2} of the latest
// residual evaluation; once sum r^2 <= tol2 * sum b^2 every later launch returns without
// touching memory. When `resid_out` is set the kernel also accumulates, in FP64, the
// residual of the iterate it reads (r = div dx^2 - (sum of neighbours - 6 p) over the
// leaf's voxels), which needs no extra memory traffic: the stencil is already staged.
//
// kNeumann: zero-gradient walls instead: a voxel's missing face neighbours take its own value,
// so it averages its n in-domain neighbours, pgs = (sum of those - div dx^2) / n (the sum in the
// order x+, x-, y+, y-, z+, z-), and the residual uses the same operator.
template <bool kNeumann>
__global__ void __launch_bounds__(kThreads) rbgs_iteration_kernel(TopoView t, const float* __restrict__ div,
                                                                   const float* __restrict__ p_in,
                                                                   float* __restrict__ p_out, float dx2, float omega,
                                                                   const double* __restrict__ check, double tol2,
                                                                   double* __restrict__ resid_out,
                                                                   unsigned long long* __restrict__ executed) {
    __shared__ float sp[PT * PT * PT];
    __shared__ float sb[RT * RT * RT];
    __shared__ int nb[27];
    __shared__ double red[2][kThreads / 32];
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int64_t leaf = blockIdx.x;
    const int tid = threadIdx.x;
    if (executed != nullptr && leaf == 0 && tid == 0) atomicAdd(executed, 1ull);
    if (tid < 27) nb[tid] = __ldg(t.nbr27 + leaf * 27 + tid);
    __syncthreads();
    for (int c = tid; c < PT * PT * PT; c += kThreads) {
        const int a = c / (PT * PT) - 2, b = (c / PT) % PT - 2, d = c % PT - 2;
        float val = 0.f;
        if (p_in != nullptr && halo_depth(a) + halo_depth(b) + halo_depth(d) <= 2) {
            const int l = nb[nbr_index(a) * 9 + nbr_index(b) * 3 + nbr_index(d)];
            if (l >= 0) val = __ldg(p_in + ((int64_t)l << 9) + local_offset(a, b, d));
        }
        sp[c] = val;
    }
    for (int c = tid; c < RT * RT * RT; c += kThreads) {
        const int a = c / (RT * RT) - 1, b = (c / RT) % RT - 1, d = c % RT - 1;
        float val = 0.f;
        if (halo_depth(a) + halo_depth(b) + halo_depth(d) <= 1) {
            const int l = nb[nbr_index(a) * 9 + nbr_index(b) * 3 + nbr_index(d)];
            if (l >= 0) val = __ldg(div + ((int64_t)l << 9) + local_offset(a, b, d));
        }
        sb[c] = val;
    }
    __syncthreads();
    if (resid_out != nullptr) {
        const double h2 = (double)dx2;
        double r2 = 0.0, b2 = 0.0;
        for (int n = tid; n < 512; n += kThreads) {
            const int a = n >> 6, b = (n >> 3) & 7, d = n & 7;
            const int q = (a + 2) * PT * PT + (b + 2) * PT + (d + 2);
            double lap;
            if constexpr (kNeumann) {
                double sum = 0.0;
                int cnt = 0;
                staged_neighbours(nb, a, b, d, [&](int off) { sum += (double)sp[q + off], ++cnt; });
                lap = sum - (double)cnt * (double)sp[q];
            } else {
                lap = (double)sp[q + PT * PT] + (double)sp[q - PT * PT] + (double)sp[q + PT] + (double)sp[q - PT] +
                      (double)sp[q + 1] + (double)sp[q - 1] - 6.0 * (double)sp[q];
            }
            const double bb = (double)sb[(a + 1) * RT * RT + (b + 1) * RT + (d + 1)] * h2;
            r2 += (bb - lap) * (bb - lap);
            b2 += bb * bb;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        if ((tid & 31) == 0) red[0][tid >> 5] = r2, red[1][tid >> 5] = b2;
        __syncthreads();
        if (tid < 32) {
            r2 = tid < kThreads / 32 ? red[0][tid] : 0.0;
            b2 = tid < kThreads / 32 ? red[1][tid] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                r2 += __shfl_xor_sync(0xffffffffu, r2, o);
                b2 += __shfl_xor_sync(0xffffffffu, b2, o);
            }
            if (tid == 0) {
                atomicAdd(resid_out, r2);
                atomicAdd(resid_out + 1, b2);
            }
        }
    }
    // Leaf origins are multiples of 8, so a voxel's colour is the parity of its local sum.
    for (int c = tid; c < RT * RT * RT; c += kThreads) {
        const int a = c / (RT * RT) - 1, b = (c / RT) % RT - 1, d = c % RT - 1;
        if (halo_depth(a) + halo_depth(b) + halo_depth(d) > 1 || ((a + b + d) & 1) != 0) continue;
        if (nb[nbr_index(a) * 9 + nbr_index(b) * 3 + nbr_index(d)] < 0) continue;
        const int q = (a + 2) * PT * PT + (b + 2) * PT + (d + 2);
        const float po = sp[q];
        sp[q] = po + omega * (relax_target<kNeumann>(sp, nb, q, a, b, d, sb[c] * dx2) - po);
    }
    __syncthreads();
    for (int n = tid; n < 512; n += kThreads) {
        const int a = n >> 6, b = (n >> 3) & 7, d = n & 7;
        if (((a + b + d) & 1) != 1) continue;
        const int q = (a + 2) * PT * PT + (b + 2) * PT + (d + 2);
        const int r = (a + 1) * RT * RT + (b + 1) * RT + (d + 1);
        const float po = sp[q];
        sp[q] = po + omega * (relax_target<kNeumann>(sp, nb, q, a, b, d, sb[r] * dx2) - po);
    }
    __syncthreads();
    for (int n = tid; n < 512; n += kThreads) {
        const int a = n >> 6, b = (n >> 3) & 7, d = n & 7;
        p_out[(leaf << 9) + n] = sp[(a + 2) * PT * PT + (b + 2) * PT + (d + 2)];
    }
}

// subtractPressureGradient (src/Cuda/Kernel.cu:495-541); sdf (or null): the collision
// treatment of the result (Kernel.cu:528-538).
// kNeumann: zero-gradient walls, a missing neighbour's pressure is the voxel's own.
template <bool kNeumann>
__global__ void __launch_bounds__(kThreads) subtract_gradient_kernel(TopoView t, const float* __restrict__ vel,
                                                                      const float* __restrict__ p,
                                                                      float* __restrict__ out, float inv_dx,
                                                                      const float* __restrict__ sdf) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float h = 0.5f * inv_dx;
    auto pn = [&](int x, int y, int z) {
        if constexpr (kNeumann) {
            const int64_t q = slot_of(t, L, x, y, z);
            return q < 0 ? __ldg(p + s) : __ldg(p + q);
        } else {
            return near_s(t, L, p, x, y, z);
        }
    };
    const float gx = (pn(i + 1, j, k) - pn(i - 1, j, k)) * h;
    const float gy = (pn(i, j + 1, k) - pn(i, j - 1, k)) * h;
    const float gz = (pn(i, j, k + 1) - pn(i, j, k - 1)) * h;
    const float3 u = ld3(vel, s);
    float3 r = make_float3(u.x - gx, u.y - gy, u.z - gz);
    if (sdf != nullptr) collide(t, L, sdf, s, i, j, k, inv_dx, 0.1f, r);
    st3(out, s, r);
}

// enforceCollisionBoundaries (src/Cuda/Kernel.cu:133-158), in place: every voxel reads only
// its own velocity.
__global__ void __launch_bounds__(kThreads) collision_enforce_kernel(TopoView t, float* __restrict__ vel,
                                                                      const float* __restrict__ sdf, float inv_dx) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    float3 u = make_float3(vel[3 * s], vel[3 * s + 1], vel[3 * s + 2]);
    collide(t, L, sdf, s, i, j, k, inv_dx, 0.1f, u);
    st3(vel, s, u);
}

// FP64 residual of the relaxed system: r = div dx^2 - (sum of 6 neighbours - 6 p).
template <bool kNeumann>
__global__ void __launch_bounds__(kThreads) residual_kernel(TopoView t, const float* __restrict__ div,
                                                             const float* __restrict__ p, double* __restrict__ acc,
                                                             double h2) {
    __shared__ LeafNbhd L;
    __shared__ double red[2][kThreads / 32];
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    double lap;
    if constexpr (kNeumann) {
        // The in-domain neighbours only (zero-gradient walls).
        const int di[6] = {1, -1, 0, 0, 0, 0}, dj[6] = {0, 0, 1, -1, 0, 0}, dk[6] = {0, 0, 0, 0, 1, -1};
        double sum = 0.0;
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int64_t ns = slot_of(t, L, i + di[q], j + dj[q], k + dk[q]);
            if (ns >= 0) sum += (double)__ldg(p + ns), ++cnt;
        }
        lap = sum - (double)cnt * (double)__ldg(p + s);
    } else {
        lap = (double)near_s(t, L, p, i + 1, j, k) + (double)near_s(t, L, p, i - 1, j, k) +
              (double)near_s(t, L, p, i, j + 1, k) + (double)near_s(t, L, p, i, j - 1, k) +
              (double)near_s(t, L, p, i, j, k + 1) + (double)near_s(t, L, p, i, j, k - 1) - 6.0 * (double)__ldg(p + s);
    }
    const double b = (double)__ldg(div + s) * h2;
    double r2 = (b - lap) * (b - lap), b2 = b * b;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        b2 += __shfl_xor_sync(0xffffffffu, b2, o);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = r2, red[1][threadIdx.x >> 5] = b2;
    __syncthreads();
    if (threadIdx.x < 32) {
        r2 = threadIdx.x < kThreads / 32 ? red[0][threadIdx.x] : 0.0;
        b2 = threadIdx.x < kThreads / 32 ? red[1][threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        if (threadIdx.x == 0) {
            atomicAdd(acc, r2);
            atomicAdd(acc + 1, b2);
        }
    }
}

// ---- forces ---------------------------------------------------------------------------------

// vorticityConfinement (src/Cuda/Kernel.cu:682-727), out of place.
__global__ void __launch_bounds__(kThreads) vorticity_kernel(TopoView t, const float* __restrict__ vel,
                                                              float* __restrict__ out, float dt, float inv_dx,
                                                              float scale, int fs) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float factor = 0.5f * inv_dx;
    const float3 px = near_v(t, L, vel, i + 1, j, k), mx = near_v(t, L, vel, i - 1, j, k);
    const float3 py = near_v(t, L, vel, i, j + 1, k), my = near_v(t, L, vel, i, j - 1, k);
    const float3 pz = near_v(t, L, vel, i, j, k + 1), mz = near_v(t, L, vel, i, j, k - 1);
    const float ox = ((py.z - my.z) - (pz.y - mz.y)) * factor;
    const float oy = ((pz.x - mz.x) - (px.z - mx.z)) * factor;
    const float oz = ((px.y - mx.y) - (py.x - my.x)) * factor;
    const float mpx = vort_mag(t, L, vel, i + fs, j, k, factor), mmx = vort_mag(t, L, vel, i - fs, j, k, factor);
    const float mpy = vort_mag(t, L, vel, i, j + fs, k, factor), mmy = vort_mag(t, L, vel, i, j - fs, k, factor);
    const float mpz = vort_mag(t, L, vel, i, j, k + fs, factor), mmz = vort_mag(t, L, vel, i, j, k - fs, factor);
    const float gx = (mpx - mmx) * 0.5f * inv_dx;
    const float gy = (mpy - mmy) * 0.5f * inv_dx;
    const float gz = (mpz - mmz) * 0.5f * inv_dx;
    const float glen = sqrtf(gx * gx + gy * gy + gz * gz) + 1e-5f;
    const float nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const float3 u = ld3(vel, s);
    const float fx = scale * (ny * oz - nz * oy), fy = scale * (nz * ox - nx * oz), fz = scale * (nx * oy - ny * ox);
    st3(out, s, make_float3(u.x + fx * dt, u.y + fy * dt, u.z + fz * dt));
}

// ---- topology queries -----------------------------------------------------------------------

__global__ void index_offsets_kernel(TopoView t, const int32_t* __restrict__ ijk, int64_t n, uint64_t* __restrict__ out) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = ijk[3 * q], j = ijk[3 * q + 1], k = ijk[3 * q + 2];
    const int l = leaf_from_table(t, i, j, k);
    out[q] = l < 0 ? 0ull : 1ull + ((uint64_t)l << 9) + (uint64_t)local_offset(i, j, k);
}

unsigned leaf_blocks(const Context& c) { return (unsigned)(c.topo.num_leaves * 2); }

}  // namespace

void launch_advect_fused(const Context& c, const float* vel, float* vel_out, const FieldSet& f, float dt, const float* sdf) {
    advect_fused_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, vel_out, f, dt * (1.0f / c.dx), sdf,
                                                                   1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_advect_scalars(const Context& c, const float* vel, const FieldSet& f, float dt, const float* sdf) {
    advect_scalars_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, f, dt * (1.0f / c.dx), sdf);
    HNS_LAUNCHED();
}

void launch_collision_enforce(const Context& c, float* vel, const float* sdf) {
    collision_enforce_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, sdf, 1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_divergence(const Context& c, const float* vel, float* div) {
    divergence_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, div, 1.0f / c.dx);
    HNS_LAUNCHED();
}

void launch_rbgs_iteration(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                           unsigned flags, const double* check, double tol2, double* resid_out) {
    if (flags & HNS_SOLVE_NEUMANN) {  // zero-gradient walls: the staged kernel's Neumann form
        rbgs_iteration_kernel<true><<<(unsigned)c.topo.num_leaves, kThreads, 0, c.stream>>>(
            c.topo.view, div, p_in, p_out, c.dx * c.dx, omega, check, tol2, resid_out, c.counters);
        HNS_LAUNCHED();
        return;
    }
    // One iteration at a time (the colour-split form runs whole solves): the staged kernel.
    if ((c.rbgs_kernel == HNS_RBGS_BULK || c.rbgs_kernel == HNS_RBGS_SPLIT) && rbgs_bulk_eligible(div, p_in, p_out)) {
        launch_rbgs_bulk(c, div, p_in, p_out, omega, check, tol2, resid_out);
        return;
    }
    rbgs_iteration_kernel<false><<<(unsigned)c.topo.num_leaves, kThreads, 0, c.stream>>>(
        c.topo.view, div, p_in, p_out, c.dx * c.dx, omega, check, tol2, resid_out, c.counters);
    HNS_LAUNCHED();
}

void launch_subtract_gradient(const Context& c, const float* vel, const float* p, float* out, const float* sdf,
                              unsigned flags) {
    if (flags & HNS_SOLVE_NEUMANN) {
        if (sdf) fail(HNS_ERR_UNSUPPORTED, "zero-gradient walls do not take a collider");
        subtract_gradient_kernel<true><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, p, out, 1.0f / c.dx,
                                                                                    nullptr);
    } else {
        subtract_gradient_kernel<false><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, p, out,
                                                                                     1.0f / c.dx, sdf);
    }
    HNS_LAUNCHED();
}

void launch_vorticity(const Context& c, const float* vel, float* out, float dt, float scale, float factor_scale) {
    vorticity_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, out, dt, 1.0f / c.dx, scale,
                                                                (int)factor_scale);
    HNS_LAUNCHED();
}

void launch_residual(const Context& c, const float* div, const float* p, double* acc, unsigned flags) {
    const double h = (double)c.dx;
    if (flags & HNS_SOLVE_NEUMANN)
        residual_kernel<true><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, div, p, acc, h * h);
    else
        residual_kernel<false><<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, div, p, acc, h * h);
    HNS_LAUNCHED();
}

void launch_index_offsets(const Context& c, const int32_t* ijk, int64_t n, uint64_t* out) {
    if (n <= 0) return;
    index_offsets_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(c.topo.view, ijk, n, out);
    HNS_LAUNCHED();
}

}  // namespace hns
