// Geometric multigrid V-cycle for the inner solve of the FP64 refinement (HNS_SOLVE_MULTIGRID):
// the preconditioner the reference declares for the projection but never implements
// (restrict_to_2x2x2 / prolongate / compute_residual / update_pressure,
// src/Cuda/Kernels.cuh:52-60).
//
// Levels live inside the leaf structure: level l has s = 8 >> l cells per leaf side (8, 4, 2, 1),
// so every level shares the leaf table and the 27-neighbour table, and a cell's face
// neighbour is in its own leaf or in the face-neighbour leaf. Cells of a leaf are stored at
// (x s + y) s + z. With unit fine spacing the level-l operator is
// A_l u = (sum of the 6 face neighbours - 6 u) / 4^l, zero outside the domain (the fine
// system's p = 0 walls). The cycle: red-black Gauss-Seidel smoothing (red by global cell
// parity), the residual, restriction by the mean of the 8 children, on down to one cell per
// leaf, where SOR sweeps solve the leaf-level system; then each coarse correction goes back
// into the fine cells, interpolated trilinearly between cell centres, and post-smoothing.
// FP32 throughout; the FP64 outer refinement around it measures the residual exactly, so the
// cycle only has to reduce the error. Every kernel returns at once when the refinement has
// converged.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "hns_internal.cuh"

namespace hns {
namespace {

constexpr int kThreads = 256;
constexpr int kLevels = 4;
// Cycle parameters: smoothing iterations before and after the coarse correction, and SOR
// iterations (factor kCoarseOmega) at the one-cell-per-leaf level.
constexpr int kPreSmooth = 3, kPostSmooth = 3, kCoarseIters = 60;
constexpr float kCoarseOmega = 1.9f;

__device__ __forceinline__ bool done(const double* check, double tol2) {
    return check != nullptr && check[0] <= tol2 * check[1];
}

// Cell q of level with 2^lg cells per leaf side: its leaf and coordinates within the leaf.
struct Cell {
    int64_t leaf;
    int x, y, z;
};

__device__ __forceinline__ Cell cell_of(int64_t q, int lg) {
    Cell c;
    c.leaf = q >> (3 * lg);
    const int loc = (int)(q & ((1 << (3 * lg)) - 1)), m = (1 << lg) - 1;
    c.x = loc >> (2 * lg);
    c.y = (loc >> lg) & m;
    c.z = loc & m;
    return c;
}

// u at (x, y, z) of leaf `leaf`, each coordinate in [-1, s]: a coordinate outside [0, s) is in
// the neighbour leaf across that face, edge or corner (0 when that leaf does not exist).
__device__ __forceinline__ float at(const TopoView& t, const float* __restrict__ u, int64_t leaf, int lg, int x, int y,
                                    int z) {
    const int s = 1 << lg;
    int dx = 0, dy = 0, dz = 0;
    if (x < 0) dx = -1, x += s;
    if (x >= s) dx = 1, x -= s;
    if (y < 0) dy = -1, y += s;
    if (y >= s) dy = 1, y -= s;
    if (z < 0) dz = -1, z += s;
    if (z >= s) dz = 1, z -= s;
    int64_t l = leaf;
    if (dx | dy | dz) {
        const int n = __ldg(t.nbr27 + leaf * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1));
        if (n < 0) return 0.f;
        l = n;
    }
    return u[(l << (3 * lg)) + (((x << lg) + y) << lg) + z];
}

__device__ __forceinline__ float nbr_sum(const TopoView& t, const float* __restrict__ u, const Cell& c, int lg) {
    return at(t, u, c.leaf, lg, c.x + 1, c.y, c.z) + at(t, u, c.leaf, lg, c.x - 1, c.y, c.z) +
           at(t, u, c.leaf, lg, c.x, c.y + 1, c.z) + at(t, u, c.leaf, lg, c.x, c.y - 1, c.z) +
           at(t, u, c.leaf, lg, c.x, c.y, c.z + 1) + at(t, u, c.leaf, lg, c.x, c.y, c.z - 1);
}

// One colour of SOR on level lg: u = (1 - omega) u + omega (sum - h2 b) / 6, h2 = 4^l.
__global__ void __launch_bounds__(kThreads) mg_smooth_kernel(TopoView t, float* u, const float* __restrict__ b, int lg,
                                                             int64_t cells, int colour, float omega, float h2,
                                                             const double* __restrict__ check, double tol2) {
    if (done(check, tol2)) return;
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= cells) return;
    const Cell c = cell_of(q, lg);
    const int4 o = t.origin[c.leaf];
    // Global cell coordinates: leaf origins are multiples of 8 fine voxels, 2^lg cells per leaf.
    const int gx = ((o.x >> 3) << lg) + c.x, gy = ((o.y >> 3) << lg) + c.y, gz = ((o.z >> 3) << lg) + c.z;
    if (((gx + gy + gz) & 1) != colour) return;
    const float g = (nbr_sum(t, u, c, lg) - h2 * __ldg(b + q)) * (1.0f / 6.0f);
    u[q] = u[q] + omega * (g - u[q]);
}

// r = b - (sum - 6 u) / h2.
__global__ void __launch_bounds__(kThreads) mg_residual_kernel(TopoView t, const float* __restrict__ u,
                                                               const float* __restrict__ b, float* __restrict__ r, int lg,
                                                               int64_t cells, float inv_h2, const double* __restrict__ check,
                                                               double tol2) {
    if (done(check, tol2)) return;
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= cells) return;
    const Cell c = cell_of(q, lg);
    r[q] = __ldg(b + q) - (nbr_sum(t, u, c, lg) - 6.0f * u[q]) * inv_h2;
}

// Coarse right-hand side: the mean of the 8 children's residuals (coarse level lg).
__global__ void __launch_bounds__(kThreads) mg_restrict_kernel(const float* __restrict__ r_fine, float* __restrict__ b,
                                                               int lg, int64_t cells, const double* __restrict__ check,
                                                               double tol2) {
    if (done(check, tol2)) return;
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= cells) return;
    const Cell c = cell_of(q, lg);
    const int lf = lg + 1;
    const int64_t base = c.leaf << (3 * lf);
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int x = 2 * c.x + (k >> 2), y = 2 * c.y + ((k >> 1) & 1), z = 2 * c.z + (k & 1);
        sum += __ldg(r_fine + base + (((x << lf) + y) << lf) + z);
    }
    b[q] = 0.125f * sum;
}

// u_fine += the coarse correction interpolated trilinearly between cell centres (fine level
// lg): along each axis a fine cell takes 3/4 of its parent and 1/4 of the parent's neighbour on
// its side (0 outside the domain).
__global__ void __launch_bounds__(kThreads) mg_prolong_kernel(TopoView t, const float* __restrict__ u_coarse,
                                                              float* __restrict__ u_fine, int lg, int64_t cells,
                                                              const double* __restrict__ check, double tol2) {
    if (done(check, tol2)) return;
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= cells) return;
    const Cell c = cell_of(q, lg);
    const int lc = lg - 1;
    const int X = c.x >> 1, Y = c.y >> 1, Z = c.z >> 1;
    const int dx = (c.x & 1) ? 1 : -1, dy = (c.y & 1) ? 1 : -1, dz = (c.z & 1) ? 1 : -1;
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int a = k >> 2, b = (k >> 1) & 1, e = k & 1;
        const float w = (a ? 0.25f : 0.75f) * (b ? 0.25f : 0.75f) * (e ? 0.25f : 0.75f);
        sum += w * at(t, u_coarse, c.leaf, lc, X + a * dx, Y + b * dy, Z + e * dz);
    }
    u_fine[q] += sum;
}

unsigned blocks(int64_t cells) { return (unsigned)((cells + kThreads - 1) / kThreads); }

}  // namespace

// One V-cycle on rhs b0 (n FP32 values, slot order) into u0 (n FP32, overwritten; starts at 0).
void mg_vcycle(Context& c, const float* b0, float* u0, const double* check, double tol2) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    const TopoView t = c.topo.view;
    float* u[kLevels];
    const float* b[kLevels];
    float* bw[kLevels];
    float* r[kLevels];
    int64_t cells[kLevels];
    for (int l = 0; l < kLevels; ++l) {
        const int lg = 3 - l;
        cells[l] = L << (3 * lg);
        r[l] = c.scratch_f32("mg_r" + std::to_string(l), (size_t)cells[l]);
        if (l == 0) {
            u[l] = u0, b[l] = b0, bw[l] = nullptr;
        } else {
            u[l] = c.scratch_f32("mg_u" + std::to_string(l), (size_t)cells[l]);
            bw[l] = c.scratch_f32("mg_b" + std::to_string(l), (size_t)cells[l]);
            b[l] = bw[l];
        }
    }
    auto smooth = [&](int l, int iters, float omega) {
        const float h2 = (float)(1 << (2 * l));
        for (int it = 0; it < iters; ++it)
            for (int colour = 0; colour < 2; ++colour) {
                mg_smooth_kernel<<<blocks(cells[l]), kThreads, 0, c.stream>>>(t, u[l], b[l], 3 - l, cells[l], colour, omega,
                                                                              h2, check, tol2);
                HNS_LAUNCHED();
            }
    };
    HNS_CUDA(cudaMemsetAsync(u0, 0, sizeof(float) * (size_t)cells[0], c.stream));
    for (int l = 0; l + 1 < kLevels; ++l) {
        if (l > 0) HNS_CUDA(cudaMemsetAsync(u[l], 0, sizeof(float) * (size_t)cells[l], c.stream));
        smooth(l, kPreSmooth, 1.0f);
        mg_residual_kernel<<<blocks(cells[l]), kThreads, 0, c.stream>>>(t, u[l], b[l], r[l], 3 - l, cells[l],
                                                                         1.0f / (float)(1 << (2 * l)), check, tol2);
        HNS_LAUNCHED();
        mg_restrict_kernel<<<blocks(cells[l + 1]), kThreads, 0, c.stream>>>(r[l], bw[l + 1], 3 - (l + 1), cells[l + 1],
                                                                             check, tol2);
        HNS_LAUNCHED();
    }
    HNS_CUDA(cudaMemsetAsync(u[kLevels - 1], 0, sizeof(float) * (size_t)cells[kLevels - 1], c.stream));
    smooth(kLevels - 1, kCoarseIters, kCoarseOmega);
    for (int l = kLevels - 2; l >= 0; --l) {
        mg_prolong_kernel<<<blocks(cells[l]), kThreads, 0, c.stream>>>(t, u[l + 1], u[l], 3 - l, cells[l], check, tol2);
        HNS_LAUNCHED();
        smooth(l, kPostSmooth, 1.0f);
    }
}

}  // namespace hns
