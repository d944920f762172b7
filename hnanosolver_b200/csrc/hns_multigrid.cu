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
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <utility>

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

// ---- V-cycle of the FP16 inner solve (colour-split fine level) ------------------------------
// Coarse levels as above (2^LG cells per leaf side, cell (x, y, z) of leaf l at
// (l << 3 LG) + ((x << LG) + y << LG) + z, FP32), with the operator corrected at the walls: the
// fine system's p = 0 sits at the ghost cell's centre, half a fine cell past the wall, and a
// coarse ghost value of 0 would put it half a coarse cell past it. The coarse ghost value is
// instead extrapolated linearly through that point, -gamma u with gamma = (2^l - 1) / (2^l + 1)
// at level l, which adds gamma to the diagonal for each missing face neighbour. A numpy model of
// the cycle on a 160^3 shell gives 0.16 per cycle with the correction against 0.54-1.1 without.
// Face neighbours come from the colour-split face table nb8 ({+x, -x, +y, -y, +z, -z, the leaf,
// 0}, a missing leaf = num_leaves).

template <int LG>
struct LevelCell {
    int leaf, x, y, z;
};

template <int LG>
__device__ __forceinline__ LevelCell<LG> level_cell(int64_t q) {
    constexpr int m = (1 << LG) - 1;
    LevelCell<LG> c;
    c.leaf = (int)(q >> (3 * LG));
    c.x = (int)(q >> (2 * LG)) & m;
    c.y = (int)(q >> LG) & m;
    c.z = (int)q & m;
    return c;
}

// Sum of the face neighbours of cell (x, y, z) of `leaf` at level LG present in the domain, and
// the number missing.
template <int LG, bool kRead = true>
__device__ __forceinline__ float level_nsum(const int4* __restrict__ nb8, const float* __restrict__ u, int leaf, int x,
                                            int y, int z, int num_leaves, int& missing) {
    constexpr int s = 1 << LG, m = s - 1;
    const int4 f0 = __ldg(nb8 + 2 * leaf), f1 = __ldg(nb8 + 2 * leaf + 1);
    auto at = [&](int l, int a, int b, int c) -> float {
        if (l >= num_leaves) {
            ++missing;
            return 0.f;
        }
        return kRead ? u[((int64_t)l << (3 * LG)) + (((a << LG) + b) << LG) + c] : 0.f;
    };
    missing = 0;
    float sum = at(x < m ? leaf : f0.x, (x + 1) & m, y, z);
    sum += at(x > 0 ? leaf : f0.y, (x - 1) & m, y, z);
    sum += at(y < m ? leaf : f0.z, x, (y + 1) & m, z);
    sum += at(y > 0 ? leaf : f0.w, x, (y - 1) & m, z);
    sum += at(z < m ? leaf : f1.x, x, y, (z + 1) & m);
    sum += at(z > 0 ? leaf : f1.y, x, y, (z - 1) & m);
    return sum;
}

// One colour of SOR at level LG: u += omega ((sum - h2 b) / (6 + gamma missing) - u). Colour:
// the global cell parity, which for LG >= 1 is that of the local coordinates (leaf origins are
// even in cells) and for LG = 0 that of the leaf.
template <int LG>
__global__ void __launch_bounds__(kThreads) mgl_smooth_kernel(TopoView t, const int4* __restrict__ nb8, float* u,
                                                              const float* __restrict__ b, int colour, int zero,
                                                              float omega, float h2, float gamma,
                                                              const double* __restrict__ check, double tol2) {
    if (done(check, tol2)) return;
    // Programmatic dependent launches: the next kernel of the cycle may be scheduled now; u and
    // b are read after griddepcontrol.wait (a no-op for an ordinary launch).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int num_leaves = (int)t.num_leaves;
    const int64_t t0 = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    LevelCell<LG> c;
    int64_t q, other = -1;
    if constexpr (LG == 0) {
        // One cell per leaf: the leaf's parity decides; from u = 0 the other colour writes 0.
        if (t0 >= num_leaves) return;
        q = t0;
        c = level_cell<0>(q);
        const int4 o = t.origin[c.leaf];
        if ((((o.x + o.y + o.z) >> 3) & 1) != colour) {
            if (zero) {
                asm volatile("griddepcontrol.wait;" ::: "memory");
                u[q] = 0.f;
            }
            return;
        }
    } else {
        // One thread per cell of the colour: the z pair (2k, 2k + 1) of row (x, y) holds one; from
        // u = 0 the thread also writes the pair's other cell.
        constexpr int m = (1 << LG) - 1, hz = (1 << (LG - 1)) - 1;
        if (t0 >= ((int64_t)num_leaves << (3 * LG - 1))) return;
        c.leaf = (int)(t0 >> (3 * LG - 1));
        c.x = (int)(t0 >> (2 * LG - 1)) & m;
        c.y = (int)(t0 >> (LG - 1)) & m;
        const int z0 = 2 * ((int)t0 & hz);
        c.z = z0 + ((c.x + c.y + colour) & 1);
        q = ((int64_t)c.leaf << (3 * LG)) + (((c.x << LG) + c.y) << LG) + c.z;
        other = q + (c.z == z0 ? 1 : -1);
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    int missing;
    if (zero) {
        // u = 0 before this sweep (the first of a level's cycle): no neighbour is read.
        float unused = level_nsum<LG, false>(nb8, u, c.leaf, c.x, c.y, c.z, num_leaves, missing);
        (void)unused;
        u[q] = omega * (-h2 * __ldg(b + q)) / (6.0f + gamma * (float)missing);
        if constexpr (LG > 0) u[other] = 0.f;
        return;
    }
    const float sum = level_nsum<LG>(nb8, u, c.leaf, c.x, c.y, c.z, num_leaves, missing);
    const float uq = u[q];
    u[q] = uq + omega * ((sum - h2 * __ldg(b + q)) / (6.0f + gamma * (float)missing) - uq);
}

// All SOR sweeps of the coarsest level (one cell per leaf) in one launch of a thread-block
// cluster, in place of two launches per sweep. CTA r of the cluster holds the cells of leaves
// [r P, r P + P) (P = ceil(L / CTAs)): their values u (and a zero past them, the value of
// a missing neighbour), right-hand sides b and a 32-byte record per cell, made once per context
// by coarse_table_kernel: the six face neighbours as (CTA rank << 16) | index in that CTA's u,
// the diagonal 6 + gamma missing, the cell's index; colour-0 records from the front of the
// table, colour-1 records from the back. Neighbours' values are read through the cluster's
// shared memory window (distributed shared memory), and a cluster barrier separates the
// colours. The arithmetic is mgl_smooth_kernel<0>'s, in its order: the values are its values.
// The cluster has 16 CTAs (a non-portable size) where the device schedules that, else 8.
constexpr int kCoarseThreads = 1024, kCoarseUnroll = 3;
constexpr int kCoarseCellBytes = 32 + 4 + 4;  // the record, u, b (plus 4 bytes: u's zero)

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// The shared::cluster address of shared::cta address `a` in the CTA of rank `rank`.
__device__ __forceinline__ uint32_t cluster_map(uint32_t a, uint32_t rank) {
    uint32_t d;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(rank));
    return d;
}

__device__ __forceinline__ float ld_cluster(uint32_t addr) {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

// The records of CTA r's cells (block r of one per CTA of the cluster), and its colour counts.
__global__ void __launch_bounds__(kCoarseThreads) coarse_table_kernel(TopoView t, const int4* __restrict__ nb8,
                                                                      uint4* __restrict__ table, int* __restrict__ counts,
                                                                      int per_cta, float gamma) {
    __shared__ int s_count[2];
    const int P = per_cta, tid = (int)threadIdx.x, r = (int)blockIdx.x;
    const int num_leaves = (int)t.num_leaves;
    const int lo = r * P, n = max(0, min(num_leaves - lo, P));
    if (tid == 0) s_count[0] = s_count[1] = 0;
    __syncthreads();
    uint4* rec = table + (size_t)2 * P * r;
    for (int i = tid; i < n; i += kCoarseThreads) {
        const int leaf = lo + i;
        const int4 f0 = nb8[2 * leaf], f1 = nb8[2 * leaf + 1];
        const int nbl[6] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y};
        uint32_t w[6];
        int missing = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int m = nbl[k];
            if (m >= num_leaves) {
                ++missing;
                w[k] = ((uint32_t)r << 16) | (uint32_t)P;
            } else {
                const int q = m / P;
                w[k] = ((uint32_t)q << 16) | (uint32_t)(m - q * P);
            }
        }
        const float d = 6.0f + gamma * (float)missing;
        const int4 o = t.origin[leaf];
        const int slot = (((o.x + o.y + o.z) >> 3) & 1) == 0 ? atomicAdd(&s_count[0], 1)
                                                               : P - 1 - atomicAdd(&s_count[1], 1);
        rec[2 * slot] = make_uint4(w[0], w[1], w[2], w[3]);
        rec[2 * slot + 1] = make_uint4(w[4], w[5], __float_as_uint(d), (uint32_t)i);
    }
    __syncthreads();
    if (tid == 0) {
        counts[2 * r] = s_count[0];
        counts[2 * r + 1] = s_count[1];
    }
}

__global__ void __launch_bounds__(kCoarseThreads, 1)
    coarsest_cluster_kernel(const uint4* __restrict__ table, const int* __restrict__ counts, float* __restrict__ u_out,
                            const float* __restrict__ b, int num_leaves, int per_cta, int sweeps, float omega, float h2,
                            const double* __restrict__ check, double tol2) {
    extern __shared__ __align__(16) unsigned char coarse_smem[];
    __shared__ float s_skip;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int P = per_cta, tid = (int)threadIdx.x;
    uint4* srec = reinterpret_cast<uint4*>(coarse_smem);
    float* su = reinterpret_cast<float*>(srec + 2 * P);  // P + 1 values, su[P] = 0
    float* sb = su + P + 1;
    const uint32_t rank = cluster_ctarank();
    const int lo = (int)rank * P, n = max(0, min(num_leaves - lo, P));
    const int c0 = __ldg(counts + 2 * rank), c1 = __ldg(counts + 2 * rank + 1);
    // The records (the topology only) before the wait on the preceding kernel.
    const uint4* g = table + (size_t)2 * P * rank;
    for (int k = tid; k < 2 * P; k += kCoarseThreads) srec[k] = __ldg(g + k);
    if (tid == 0) {
        su[P] = 0.f;
        s_skip = 0.f;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (rank == 0 && tid == 0 && done(check, tol2)) s_skip = 1.f;
    for (int i = tid; i < n; i += kCoarseThreads) sb[i] = __ldg(b + lo + i);
    cluster_barrier();
    // Every CTA takes rank 0's decision, so all or none reach the sweeps' barriers; rank 0's
    // memory stays until each has read it.
    if (ld_cluster(cluster_map((uint32_t)__cvta_generic_to_shared(&s_skip), 0)) != 0.f) {
        cluster_barrier();
        return;
    }
    const uint32_t su_addr = (uint32_t)__cvta_generic_to_shared(su);
    for (int it = 0; it < sweeps; ++it) {
        for (int colour = 0; colour < 2; ++colour) {
            const int begin = colour ? P - c1 : 0, end = colour ? P : c0;
            if (it == 0 && colour == 0) {
                // u = 0 before this sweep: no neighbour is read, the other colour is set to 0.
                for (int j = begin + tid; j < end; j += kCoarseThreads) {
                    const uint4 q = srec[2 * j + 1];
                    su[q.w] = omega * (-h2 * sb[q.w]) / __uint_as_float(q.z);
                }
                for (int j = P - c1 + tid; j < P; j += kCoarseThreads) su[srec[2 * j + 1].w] = 0.f;
            } else {
                // kCoarseUnroll cells per thread at a time: every load issued before the first use.
                for (int j0 = begin + tid; j0 < end; j0 += kCoarseUnroll * kCoarseThreads) {
                    uint4 qa[kCoarseUnroll], qb[kCoarseUnroll];
                    float v[kCoarseUnroll][6];
#pragma unroll
                    for (int k = 0; k < kCoarseUnroll; ++k) {
                        const int j = j0 + k * kCoarseThreads;
                        if (j < end) {
                            qa[k] = srec[2 * j];
                            qb[k] = srec[2 * j + 1];
                        }
                    }
#pragma unroll
                    for (int k = 0; k < kCoarseUnroll; ++k) {
                        if (j0 + k * kCoarseThreads < end) {
                            const uint32_t w[6] = {qa[k].x, qa[k].y, qa[k].z, qa[k].w, qb[k].x, qb[k].y};
#pragma unroll
                            for (int e = 0; e < 6; ++e)
                                v[k][e] = ld_cluster(cluster_map(su_addr + ((w[e] & 0xffffu) << 2), w[e] >> 16));
                        }
                    }
#pragma unroll
                    for (int k = 0; k < kCoarseUnroll; ++k) {
                        if (j0 + k * kCoarseThreads < end) {
                            float sum = v[k][0];
                            sum += v[k][1];
                            sum += v[k][2];
                            sum += v[k][3];
                            sum += v[k][4];
                            sum += v[k][5];
                            const uint32_t i = qb[k].w;
                            const float uq = su[i];
                            su[i] = uq + omega * ((sum - h2 * sb[i]) / __uint_as_float(qb[k].z) - uq);
                        }
                    }
                }
            }
            cluster_barrier();
        }
    }
    // After the last barrier no CTA reads another's memory.
    for (int i = tid; i < n; i += kCoarseThreads) u_out[lo + i] = su[i];
}

// The same sweep at level 1 (4^3 cells per leaf) by rows: one thread per z-row (4 contiguous
// floats), which updates its 2 cells of the colour from 16-byte loads of the row, its right-hand
// side and its 4 x/y neighbour rows (across a face, the neighbour leaf's row; a missing leaf adds
// gamma to the diagonal) and the values past its z ends, and stores the row back whole (no other
// thread writes it in this sweep). Neighbours are summed in mgl_smooth_kernel's order, so the
// values are its values: 8 loads for 2 updates where it makes 20.
__global__ void __launch_bounds__(kThreads) level1_smooth_rows_kernel(const int4* __restrict__ nb8, float* u,
                                                                      const float* __restrict__ b, int num_leaves,
                                                                      int colour, int zero, float omega, float h2,
                                                                      float gamma, const double* __restrict__ check,
                                                                      double tol2) {
    if (done(check, tol2)) return;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int64_t tid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (tid >= ((int64_t)num_leaves << 4)) return;
    const int leaf = (int)(tid >> 4), x = (int)(tid >> 2) & 3, y = (int)tid & 3;
    const int4 f0 = __ldg(nb8 + 2 * leaf), f1 = __ldg(nb8 + 2 * leaf + 1);
    auto row_of = [&](int l, int a, int c2) { return ((int64_t)l << 6) + (((a << 2) + c2) << 2); };
    const int lxp = x < 3 ? leaf : f0.x, lxm = x > 0 ? leaf : f0.y, lyp = y < 3 ? leaf : f0.z, lym = y > 0 ? leaf : f0.w;
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    auto ld4 = [&](int l, int64_t off) { return l < num_leaves ? __ldg(reinterpret_cast<const float4*>(u + off)) : z4; };
    const int64_t own = row_of(leaf, x, y);
    const float4 bb = __ldg(reinterpret_cast<const float4*>(b + own));
    float4 c4 = zero ? z4 : __ldg(reinterpret_cast<const float4*>(u + own));
    const float4 xp = zero ? z4 : ld4(lxp, row_of(lxp, (x + 1) & 3, y));
    const float4 xm = zero ? z4 : ld4(lxm, row_of(lxm, (x - 1) & 3, y));
    const float4 yp = zero ? z4 : ld4(lyp, row_of(lyp, x, (y + 1) & 3));
    const float4 ym = zero ? z4 : ld4(lym, row_of(lym, x, (y - 1) & 3));
    const float zhi = (zero || f1.x >= num_leaves) ? 0.f : __ldg(u + row_of(f1.x, x, y));
    const float zlo = (zero || f1.y >= num_leaves) ? 0.f : __ldg(u + row_of(f1.y, x, y) + 3);
    const int lateral = (lxp >= num_leaves) + (lxm >= num_leaves) + (lyp >= num_leaves) + (lym >= num_leaves);
    float cv[4] = {c4.x, c4.y, c4.z, c4.w};
    const float bv[4] = {bb.x, bb.y, bb.z, bb.w};
    const float xpv[4] = {xp.x, xp.y, xp.z, xp.w}, xmv[4] = {xm.x, xm.y, xm.z, xm.w};
    const float ypv[4] = {yp.x, yp.y, yp.z, yp.w}, ymv[4] = {ym.x, ym.y, ym.z, ym.w};
    const float old[4] = {cv[0], cv[1], cv[2], cv[3]};
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        if (((x + y + z) & 1) != colour) continue;  // the other colour keeps its value (0 from zero)
        const int missing = lateral + (z == 3 && f1.x >= num_leaves) + (z == 0 && f1.y >= num_leaves);
        const float diag = 6.0f + gamma * (float)missing;
        if (zero) {
            cv[z] = omega * (-h2 * bv[z]) / diag;
        } else {
            float sum = xpv[z];
            sum += xmv[z];
            sum += ypv[z];
            sum += ymv[z];
            sum += z < 3 ? old[z < 3 ? z + 1 : 3] : zhi;
            sum += z > 0 ? old[z > 0 ? z - 1 : 0] : zlo;
            cv[z] = old[z] + omega * ((sum - h2 * bv[z]) / diag - old[z]);
        }
    }
    *reinterpret_cast<float4*>(u + own) = make_float4(cv[0], cv[1], cv[2], cv[3]);
}

// bc (level LG - 1) = the mean of the residuals b - (sum - (6 + gamma missing) u) / h2 of each
// coarse cell's 8 children at level LG.
template <int LG>
__global__ void __launch_bounds__(kThreads) mgl_restrict_kernel(const int4* __restrict__ nb8, const float* __restrict__ u,
                                                                const float* __restrict__ b, float* __restrict__ bc,
                                                                int num_leaves, float inv_h2, float gamma,
                                                                const double* __restrict__ check, double tol2) {
    if (done(check, tol2)) return;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= ((int64_t)num_leaves << (3 * (LG - 1)))) return;
    const LevelCell<LG - 1> cc = level_cell<LG - 1>(q);
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int x = 2 * cc.x + (k >> 2), y = 2 * cc.y + ((k >> 1) & 1), z = 2 * cc.z + (k & 1);
        const int64_t f = ((int64_t)cc.leaf << (3 * LG)) + (((x << LG) + y) << LG) + z;
        int missing;
        const float ns = level_nsum<LG>(nb8, u, cc.leaf, x, y, z, num_leaves, missing);
        sum += __ldg(b + f) - (ns - (6.0f + gamma * (float)missing) * u[f]) * inv_h2;
    }
    bc[q] = 0.125f * sum;
}

// Prolongation, one thread per coarse cell (level LC, 2^LC cells per leaf side): the coarse
// correction at the cell and its 26 neighbours (across faces, edges and corners of the leaf from
// the 27-neighbour table, 0 outside the domain), then each of the cell's 8 children at level
// LC + 1 takes the trilinear interpolation between cell centres: along each axis 3/4 of the
// parent and 1/4 of the parent's neighbour on the child's side.
template <int LC>
__device__ __forceinline__ void gather27(const TopoView& t, const float* __restrict__ uc, int leaf, int X, int Y, int Z,
                                         float v[27]) {
    constexpr int sc = 1 << LC;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        int cx = X + k / 9 - 1, cy = Y + (k / 3) % 3 - 1, cz = Z + k % 3 - 1;
        const int ox = cx < 0 ? -1 : (cx >= sc ? 1 : 0), oy = cy < 0 ? -1 : (cy >= sc ? 1 : 0),
                  oz = cz < 0 ? -1 : (cz >= sc ? 1 : 0);
        int l = leaf;
        if (ox | oy | oz) l = __ldg(t.nbr27 + (int64_t)leaf * 27 + (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1));
        cx -= ox * sc, cy -= oy * sc, cz -= oz * sc;
        v[k] = l < 0 ? 0.f : __ldg(uc + ((int64_t)l << (3 * LC)) + (((cx << LC) + cy) << LC) + cz);
    }
}

// The interpolated value of child (i, j, k) (each 0 or 1) from the gathered neighbourhood.
__device__ __forceinline__ float interp8(const float v[27], int i, int j, int k) {
    const int sx = i ? 1 : -1, sy = j ? 1 : -1, sz = k ? 1 : -1;
    float sum = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int a = q >> 2, bb = (q >> 1) & 1, e = q & 1;
        const float w = (a ? 0.25f : 0.75f) * (bb ? 0.25f : 0.75f) * (e ? 0.25f : 0.75f);
        sum += w * v[(1 + a * sx) * 9 + (1 + bb * sy) * 3 + (1 + e * sz)];
    }
    return sum;
}

// Position of local voxel (x, y, z) of leaf l in the colour-split FP16 layout of the inner solve
// (a leaf's colour-0 values, then its colour-1 values; row (x, y) at R = 32 ((x + y) & 1) + 4 x +
// (y >> 1) within a colour, entry z >> 1 of the row).
__device__ __forceinline__ uint32_t split_at(int l, int x, int y, int z) {
    return ((uint32_t)l << 9) | ((uint32_t)((x + y + z) & 1) << 8) |
           (uint32_t)(4 * (32 * ((x + y) & 1) + 4 * x + (y >> 1)) + (z >> 1));
}

__device__ __forceinline__ float h16(const __half* p, uint32_t i) { return __half2float(p[i]); }

// The 8 values of row (x, y) of leaf l, z order, from its two colour blocks (colour c holds
// z = 2 j + ((x + y + c) & 1) at entries 4 R + j).
__device__ __forceinline__ void row8(const __half* p, int l, int x, int y, float v[8]) {
    const uint32_t R = (uint32_t)(32 * ((x + y) & 1) + 4 * x + (y >> 1));
    const uint2 a = *reinterpret_cast<const uint2*>(p + ((uint32_t)l << 9) + 4 * R);
    const uint2 b = *reinterpret_cast<const uint2*>(p + ((uint32_t)l << 9) + 256 + 4 * R);
    const int p0 = (x + y) & 1;
    const uint32_t ha[4] = {a.x & 0xFFFFu, a.x >> 16, a.y & 0xFFFFu, a.y >> 16};
    const uint32_t hb[4] = {b.x & 0xFFFFu, b.x >> 16, b.y & 0xFFFFu, b.y >> 16};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float fa = __half2float(__ushort_as_half((unsigned short)ha[j]));
        const float fb = __half2float(__ushort_as_half((unsigned short)hb[j]));
        v[2 * j] = p0 ? fb : fa;
        v[2 * j + 1] = p0 ? fa : fb;
    }
}

// Fine level of the FP16 cycle: b1 (4^3 cells per leaf) = the mean of the residuals
// r^ - (sum - 6 e) (unit spacing; a missing leaf is the zero leaf past the last one, p = 0 outside
// the domain) of each level-1 cell's 8 voxels, e and r^ in the colour-split layout. One thread
// per fine row (thread leaf * 64 + 8 x + y): its 8 residuals from the row, its four neighbour
// rows (across a face: the neighbour leaf's row) and the two values past its z ends, summed in
// z pairs; the four rows of a level-1 column (lanes differing in bits 0 and 3) are added with
// two shuffles and the column's 4 values stored by its first row.
__global__ void __launch_bounds__(kThreads) mg16_restrict_kernel(const int4* __restrict__ nb8, const __half* e,
                                                                 const __half* __restrict__ rhat, float* __restrict__ b1,
                                                                 int num_leaves, const double* __restrict__ check,
                                                                 double tol2) {
    if (done(check, tol2)) return;
    const int64_t tid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (tid >= ((int64_t)num_leaves << 6)) return;  // whole warps: 64 threads per leaf
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int leaf = (int)(tid >> 6), x = (int)(tid >> 3) & 7, y = (int)tid & 7;
    const int4 f0 = __ldg(nb8 + 2 * leaf), f1 = __ldg(nb8 + 2 * leaf + 1);
    asm volatile("griddepcontrol.wait;" ::: "memory");  // e is the preceding half-sweep's
    float c[8], xp[8], xm[8], yp[8], ym[8], rh[8];
    row8(e, leaf, x, y, c);
    row8(e, x < 7 ? leaf : f0.x, (x + 1) & 7, y, xp);
    row8(e, x > 0 ? leaf : f0.y, (x - 1) & 7, y, xm);
    row8(e, y < 7 ? leaf : f0.z, x, (y + 1) & 7, yp);
    row8(e, y > 0 ? leaf : f0.w, x, (y - 1) & 7, ym);
    row8(rhat, leaf, x, y, rh);
    const float zlo = h16(e, split_at(f1.y, x, y, 7)), zhi = h16(e, split_at(f1.x, x, y, 0));
    float part[4];
#pragma unroll
    for (int Z = 0; Z < 4; ++Z) {
        float sum = 0.f;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int z = 2 * Z + k;
            const float zm = z > 0 ? c[z > 0 ? z - 1 : 0] : zlo, zpv = z < 7 ? c[z < 7 ? z + 1 : 7] : zhi;
            sum += rh[z] - (xp[z] + xm[z] + yp[z] + ym[z] + zpv + zm - 6.0f * c[z]);
        }
        part[Z] = sum;
    }
#pragma unroll
    for (int Z = 0; Z < 4; ++Z) {
        part[Z] += __shfl_xor_sync(0xffffffffu, part[Z], 1);
        part[Z] += __shfl_xor_sync(0xffffffffu, part[Z], 8);
    }
    if (((x | y) & 1) == 0)
        *reinterpret_cast<float4*>(b1 + ((int64_t)leaf << 6) + ((((x >> 1) << 2) + (y >> 1)) << 2)) =
            make_float4(0.125f * part[0], 0.125f * part[1], 0.125f * part[2], 0.125f * part[3]);
}

// e (FP16, colour-split) += the level-1 correction interpolated trilinearly, one rounding per
// value. One thread per fine row (x, y), both colours: the 4 voxels of colour c are z = 2 j + p
// (p = (x + y + c) & 1), 8 contiguous bytes at the row's position R in the colour block; their
// parents are level-1 cells Z = j, and along z each takes 3/4 of the parent and 1/4 of Z - 1
// (p = 0) or Z + 1 (p = 1). Both colours use the 4 level-1 columns (X + {0, sx}) x (Y + {0, sy})
// (4 contiguous floats each, in this leaf or its x, y or xy-edge neighbour) and one value past
// each column's z ends (in the z neighbours of that leaf); 0 where a leaf is missing. Threads
// take consecutive R, so a warp's p is uniform.
template <int P>
__device__ __forceinline__ uint2 prolong_row(const float (&col)[2][2][4], const float (&lo)[2][2], const float (&hi)[2][2],
                                             uint2 raw) {
    uint32_t h[4] = {raw.x & 0xFFFFu, raw.x >> 16, raw.y & 0xFFFFu, raw.y >> 16};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float sum = 0.f;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const float other = P ? (j < 3 ? col[a][b][j + 1] : hi[a][b]) : (j > 0 ? col[a][b][j - 1] : lo[a][b]);
                const float w = (a ? 0.25f : 0.75f) * (b ? 0.25f : 0.75f);
                sum = fmaf(w, fmaf(0.25f, other, 0.75f * col[a][b][j]), sum);
            }
        h[j] = __half_as_ushort(__float2half_rn(__half2float(__ushort_as_half((unsigned short)h[j])) + sum));
    }
    return make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
}

__global__ void __launch_bounds__(kThreads) mg16_prolong_kernel(TopoView t, const float* __restrict__ u1, __half* e,
                                                                const double* __restrict__ check, double tol2) {
    if (done(check, tol2)) return;
    const int64_t tid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (tid >= (t.num_leaves << 6)) return;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int leaf = (int)(tid >> 6), R = (int)tid & 63;
    const int par = R >> 5, x = (R & 31) >> 2, y = 2 * (R & 3) + ((par + x) & 1);
    const int X = x >> 1, Y = y >> 1, sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1;
    const int* nb = t.nbr27 + (int64_t)leaf * 27;
    float col[2][2][4], lo[2][2], hi[2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            int cx = X + a * sx, cy = Y + b * sy;
            const int ox = cx < 0 ? -1 : (cx > 3 ? 1 : 0), oy = cy < 0 ? -1 : (cy > 3 ? 1 : 0);
            cx -= 4 * ox, cy -= 4 * oy;
            const int k = (ox + 1) * 9 + (oy + 1) * 3 + 1;  // nbr27 index of the column's leaf
            const int l = (ox | oy) ? __ldg(nb + k) : leaf, lm = __ldg(nb + k - 1), lp = __ldg(nb + k + 1);
            const int64_t off = ((cx << 2) + cy) << 2;
            const float4 v = l < 0 ? make_float4(0.f, 0.f, 0.f, 0.f)
                                   : __ldg(reinterpret_cast<const float4*>(u1 + ((int64_t)l << 6) + off));
            col[a][b][0] = v.x, col[a][b][1] = v.y, col[a][b][2] = v.z, col[a][b][3] = v.w;
            lo[a][b] = lm < 0 ? 0.f : __ldg(u1 + ((int64_t)lm << 6) + off + 3);
            hi[a][b] = lp < 0 ? 0.f : __ldg(u1 + ((int64_t)lp << 6) + off);
        }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        uint2* row = reinterpret_cast<uint2*>(e + ((uint32_t)leaf << 9) + ((uint32_t)c << 8) + 4 * R);
        *row = ((par + c) & 1) ? prolong_row<1>(col, lo, hi, *row) : prolong_row<0>(col, lo, hi, *row);
    }
}

// u (level LG) += the correction uc (level LG - 1), one thread per coarse cell.
template <int LG>
__global__ void __launch_bounds__(kThreads) mgl_prolong_kernel(TopoView t, const float* __restrict__ uc,
                                                               float* __restrict__ u, const double* __restrict__ check,
                                                               double tol2) {
    if (done(check, tol2)) return;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= (t.num_leaves << (3 * (LG - 1)))) return;
    const LevelCell<LG - 1> c = level_cell<LG - 1>(q);
    float v[27];
    gather27<LG - 1>(t, uc, c.leaf, c.x, c.y, c.z, v);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int i = k >> 2, j = (k >> 1) & 1, l = k & 1;
        const int64_t f = ((int64_t)c.leaf << (3 * LG)) + ((((2 * c.x + i) << LG) + 2 * c.y + j) << LG) + 2 * c.z + l;
        u[f] += interp8(v, i, j, l);
    }
}

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

// One V-cycle of the FP16 inner solve L e = r^ (unit spacing) on the colour-split layout: e is
// refined in place (e_zero: e = 0 before the cycle). Fine level: kMgNu red-black iterations of
// the colour-split half-sweep at omega = 1 before and after the coarse correction; levels with
// 4, 2 and 1 cells per leaf side in FP32 with the wall-corrected operator, kMgNu iterations
// before and after at the first two, SOR sweeps at the last (coarsest_schedule).
namespace {
constexpr int kMgNu = 2;

// SOR sweeps and factor at the coarsest level (one cell per leaf), from how many leaves deep the
// domain is (D, max_leaf_depth): clamp(2 D + 2, 10, 20) sweeps at clamp(2 / (1 + sin(pi / 2 D)),
// 1.5, 1.75), the optimal SOR factor for an extent of 2 D cells. Measured (ms per step, cycles
// per solve 6 on the shell, 8-10 on the fire): shell512 (D = 4) 10 at 1.5: 3.90, 20 at 1.5: 4.17,
// 5 at 1.5: 3.76 (2 doubled the cycles); fire1024 (D = 15) 10 at 1.5: 29.9, 5 at 1.5: 41 with a
// solve above the tolerance at the outer cap, 20 at 1.5: 24.3, 20 at 1.75: 21.3, 40 at 1.8: 22.0.
void coarsest_schedule(Context& c, int& sweeps, float& omega) {
    const int d = std::max(1, max_leaf_depth(c));
    sweeps = std::min(20, std::max(10, 2 * d + 2));
    omega = std::min(1.75f, std::max(1.5f, 2.0f / (1.0f + std::sin(3.14159265f / (2.0f * (float)d)))));
}

// Kernels of the cycle are programmatic dependent launches: each lets the next be scheduled
// at its start and reads the data the preceding ones wrote after griddepcontrol.wait.
template <typename... KArgs, typename... Args>
void launch_pdl(const Context& c, void (*kern)(KArgs...), int64_t threads, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks(threads));
    cfg.blockDim = dim3(kThreads);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c.add_inner_window(attr, 1);
    HNS_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
    HNS_LAUNCHED();
}

// iters red-black iterations at level l (2^LG cells per leaf side); from_zero: u = 0 before them
// (the first red sweep writes both colours).
template <int LG>
void smooth_level(Context& c, const int4* nb8, float* u, const float* b, int iters, float omega, int l, bool from_zero,
                  const double* check, double tol2) {
    const float h2 = (float)(1 << (2 * l)), gamma = (float)((1 << l) - 1) / (float)((1 << l) + 1);
    int64_t threads = c.topo.num_leaves;  // LG = 0: one thread per leaf
    if constexpr (LG > 0) threads <<= 3 * LG - 1;  // one thread per cell of the colour
    for (int it = 0; it < iters; ++it)
        for (int colour = 0; colour < 2; ++colour) {
            const int zero = (int)(from_zero && it == 0 && colour == 0);
            if constexpr (LG == 2)
                launch_pdl(c, level1_smooth_rows_kernel, c.topo.num_leaves << 4, nb8, u, b, (int)c.topo.num_leaves,
                           colour, zero, omega, h2, gamma, check, tol2);
            else
                launch_pdl(c, mgl_smooth_kernel<LG>, threads, c.topo.view, nb8, u, b, colour, zero, omega, h2, gamma,
                           check, tol2);
        }
}

}  // namespace

// Settings shared by the contexts of a process on one device (raise_device_setting).
size_t raise_device_setting(int device, int which, size_t value) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, size_t> in_force;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = in_force[{device, which}];
    if (value <= cur) return cur;
    if (which == 0)
        HNS_CUDA(cudaFuncSetAttribute(coarsest_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)value));
    else
        HNS_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, value));
    cur = value;
    return cur;
}

namespace {
// The coarsest level's `sweeps` SOR sweeps from u = 0 (level 3, one cell per leaf): one cluster
// launch where the option allows it, the leaves fit the cluster's shared memory and the device
// can schedule the cluster, else two launches per sweep. Both give the same values.
void coarsest_solve(Context& c, const int4* nb8, float* u, const float* b, int sweeps, float omega,
                    const double* check, double tol2) {
    const int64_t L = c.topo.num_leaves;
    const float h2 = 64.0f, gamma = 7.0f / 9.0f;  // level 3: (2^3)^2, (2^3 - 1) / (2^3 + 1)
    auto per_cta = [&](int ctas) { return (L + ctas - 1) / ctas; };
    auto smem_of = [&](int ctas) { return (size_t)per_cta(ctas) * kCoarseCellBytes + 4; };
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[2];
    auto configure = [&](int ctas) {
        cfg.gridDim = dim3(ctas);
        cfg.blockDim = dim3(kCoarseThreads);
        cfg.dynamicSmemBytes = smem_of(ctas);
        cfg.stream = c.stream;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    };
    bool fresh = false;
    if (c.coarse_solve == HNS_COARSE_CLUSTER && sweeps >= 1 && c.coarse_cluster_ok != 0 &&
        (c.coarse_cluster_ok < 0 || c.coarse_table_leaves != L)) {
        // The cluster size: the larger of 16 and 8 that holds the level and that the device schedules.
        c.coarse_cluster_ok = 0;
        int optin = 0;
        HNS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
        HNS_CUDA(cudaFuncSetAttribute(coarsest_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        for (int ctas : {16, 8}) {
            if (smem_of(ctas) + 16 > (size_t)optin) continue;  // + the kernel's static shared memory
            raise_device_setting(c.device, 0, smem_of(ctas));
            configure(ctas);
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, coarsest_cluster_kernel, &cfg) != cudaSuccess) {
                (void)cudaGetLastError();  // not schedulable at this size: try the next
                continue;
            }
            if (clusters >= 1) {
                c.coarse_cluster_ok = ctas;
                break;
            }
        }
        if (c.coarse_cluster_ok > 0) {
            const int ctas = c.coarse_cluster_ok;
            auto* table = reinterpret_cast<uint4*>(c.scratch_f32("mg16_coarse_records", (size_t)8 * L + 8 * ctas));
            auto* counts = reinterpret_cast<int*>(c.scratch_f32("mg16_coarse_counts", 2 * 16));
            coarse_table_kernel<<<ctas, kCoarseThreads, 0, c.stream>>>(c.topo.view, nb8, table, counts,
                                                                       (int)per_cta(ctas), gamma);
            HNS_LAUNCHED();
            if (!c.stream_capturing()) c.coarse_table_leaves = L;
            fresh = true;
        }
    }
    if (c.coarse_solve != HNS_COARSE_CLUSTER || sweeps < 1 || c.coarse_cluster_ok <= 0) {
        smooth_level<0>(c, nb8, u, b, sweeps, omega, 3, true, check, tol2);
        return;
    }
    const int ctas = c.coarse_cluster_ok;
    configure(ctas);
    // The kernel reads its records before griddepcontrol.wait: after a table made in this call,
    // an ordinary launch.
    cfg.numAttrs = fresh ? 1 : 2;
    const auto* table = reinterpret_cast<const uint4*>(c.scratch_f32("mg16_coarse_records", (size_t)8 * L + 8 * ctas));
    const auto* counts = reinterpret_cast<const int*>(c.scratch_f32("mg16_coarse_counts", 2 * 16));
    HNS_CUDA(cudaLaunchKernelEx(&cfg, coarsest_cluster_kernel, table, counts, u, b, (int)L, (int)per_cta(ctas), sweeps,
                                omega, h2, check, tol2));
    HNS_LAUNCHED();
}
}  // namespace

void mg16_vcycle(Context& c, const int* nb8, const void* rhat, void* e, bool e_zero, const double* check, double tol2) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    const TopoView t = c.topo.view;
    const auto* f8 = reinterpret_cast<const int4*>(nb8);
    const auto* r = static_cast<const __half*>(rhat);
    auto* eh = static_cast<__half*>(e);
    float* u[4] = {nullptr, nullptr, nullptr, nullptr};
    float* b[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int l = 1; l < 4; ++l) {
        const size_t cells = (size_t)L << (3 * (3 - l));
        u[l] = c.scratch_f32("mg16_u" + std::to_string(l), cells);
        b[l] = c.scratch_f32("mg16_b" + std::to_string(l), cells);
    }
    auto fine = [&](bool zero_first) {
        for (int it = 0; it < kMgNu; ++it) {
            launch_rbgs_split_half(c, nb8, rhat, e, 0, zero_first && it == 0, 1.0f, check, tol2, false);
            launch_rbgs_split_half(c, nb8, rhat, e, 1, false, 1.0f, check, tol2, false);
        }
    };
    fine(e_zero);
    launch_pdl(c, mg16_restrict_kernel, L << 6, f8, (const __half*)eh, r, b[1], (int)L, check, tol2);
    smooth_level<2>(c, f8, u[1], b[1], kMgNu, 1.0f, 1, true, check, tol2);
    launch_pdl(c, mgl_restrict_kernel<2>, L << 3, f8, (const float*)u[1], (const float*)b[1], b[2], (int)L, 0.25f,
               1.0f / 3.0f, check, tol2);
    smooth_level<1>(c, f8, u[2], b[2], kMgNu, 1.0f, 2, true, check, tol2);
    launch_pdl(c, mgl_restrict_kernel<1>, L, f8, (const float*)u[2], (const float*)b[2], b[3], (int)L, 1.0f / 16.0f,
               0.6f, check, tol2);
    int coarse_sweeps;
    float coarse_omega;
    coarsest_schedule(c, coarse_sweeps, coarse_omega);
    coarsest_solve(c, f8, u[3], b[3], coarse_sweeps, coarse_omega, check, tol2);
    launch_pdl(c, mgl_prolong_kernel<1>, L, t, (const float*)u[3], u[2], check, tol2);
    smooth_level<1>(c, f8, u[2], b[2], kMgNu, 1.0f, 2, false, check, tol2);
    launch_pdl(c, mgl_prolong_kernel<2>, L << 3, t, (const float*)u[2], u[1], check, tol2);
    smooth_level<2>(c, f8, u[1], b[1], kMgNu, 1.0f, 1, false, check, tol2);
    launch_pdl(c, mg16_prolong_kernel, L << 6, t, (const float*)u[1], eh, check, tol2);
    fine(false);
}

}  // namespace hns
