// The red-black SOR iteration, staged with bulk async copies.
//
// One CTA per 8^3 leaf performs one full iteration of redBlackGaussSeidelUpdate
// (src/Cuda/Kernel.cu:459-489) -- red on the leaf and its one-voxel face ring, then black
// on the leaf -- from p_in to p_out, reading p with a two-voxel halo and div with a
// one-voxel halo, as rbgs_iteration_kernel in hns_kernels.cu does. What differs is how the
// stencil reaches shared memory:
//
//   * Shared memory holds z-rows of 8 values. A leaf's slot order is x-major
//     (x*64 + y*8 + z), so every x-plane of a leaf (64 values), every pair of y-rows of a
//     plane (16 values) and every single row (8 values) is contiguous in HBM and lands
//     contiguously in the row layout. Those pieces -- 8 interior planes, the x-face planes,
//     the y-face rows and the xy-edge rows of p and div, 58 copies of 32..256 bytes -- are
//     fetched by cp.async.bulk, issued by one warp and counted on one mbarrier.
//   * The z-halo (values at z = -2, -1, 8, 9 of a row) is not contiguous in HBM (one or two
//     values per 32-byte row); it is fetched with plain loads into separate arrays while
//     the bulk copies are in flight.
//   * Red and black voxels are enumerated compactly (no idle iterations), and the leaf is
//     stored back with coalesced 16-byte stores.
//
// Arithmetic, order of the six-neighbour sum and the Dirichlet-0 walls are those of the
// reference; results equal rbgs_iteration_kernel's to the bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "hns_internal.cuh"
#include "hns_ptx.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

constexpr uint32_t kMaxPolls = 1u << 22;  // bounded mbarrier wait (far above any real copy latency)

// Neighbour-table index of the leaf at offset (dx, dy, dz) in {-1,0,1}^3.
__host__ __device__ constexpr int nbi(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }

struct Smem {
    float P[12 * 12 * 8];   // p rows: (a+2, b+2) for a, b in [-2, 9], z in [0, 8)
    float B[10 * 10 * 8];   // div rows: (a+1, b+1) for a, b in [-1, 8]
    float PZ[12 * 12 * 4];  // p at z = -2, -1, 8, 9 of row (a+2, b+2)
    float BZ[8 * 8 * 2];    // div at z = -1, 8 of interior row (a, b)
    double red[2][8];
    uint64_t bar;
    int nb[27];
};

__device__ __forceinline__ int prow(int a, int b) { return (a + 2) * 12 + (b + 2); }
__device__ __forceinline__ int brow(int a, int b) { return (a + 1) * 10 + (b + 1); }

// Value of p at local (a, b, d), d in [-2, 9].
__device__ __forceinline__ float pv(const Smem& s, int a, int b, int d) {
    const int r = prow(a, b);
    if ((unsigned)d < 8u) return s.P[r * 8 + d];
    return s.PZ[r * 4 + (d < 0 ? d + 2 : d - 6)];
}

__device__ __forceinline__ float bv(const Smem& s, int a, int b, int d) {
    if ((unsigned)d < 8u) return s.B[brow(a, b) * 8 + d];
    return s.BZ[(a * 8 + b) * 2 + (d < 0 ? 0 : 1)];
}

// One SOR update at (a, b, d), d in [0, 8), of a row whose x/y neighbour rows are staged (the
// leaf's rows and the x/y ring rows), in the reference's neighbour order (x+, x-, y+, y-,
// z+, z-). A row's p index is r*8 + d with r = prow(a, b); neighbour rows are r +- 12
// (x) and r +- 1 (y); the z-halo of the row is PZ[r*4 + 1] (z = -1) and PZ[r*4 + 2] (z = 8).
__device__ __forceinline__ void relax_row(Smem& s, int r, int rb, int d, float dx2, float omega) {
    const float* P = s.P;
    const int c = r * 8 + d;
    const float zp = d < 7 ? P[c + 1] : s.PZ[r * 4 + 2];
    const float zm = d > 0 ? P[c - 1] : s.PZ[r * 4 + 1];
    const float sum = P[c + 96] + P[c - 96] + P[c + 8] + P[c - 8] + zp + zm;
    const float pgs = (sum - s.B[rb * 8 + d] * dx2) * dev::kInv6;
    const float po = P[c];
    s.P[c] = po + omega * (pgs - po);
}

// The same update at a z-ring voxel (a, b, -1) or (a, b, 8) with a, b in [0, 8): the voxel and
// its x/y neighbours live in the z-halo arrays.
__device__ __forceinline__ void relax_zring(Smem& s, int a, int b, int hi, float dx2, float omega) {
    const int r = prow(a, b), k = hi ? 2 : 1;
    const float* Z = s.PZ;
    const float zp = hi ? Z[r * 4 + 3] : s.P[r * 8 + 0];
    const float zm = hi ? s.P[r * 8 + 7] : Z[r * 4 + 0];
    const float sum = Z[(r + 12) * 4 + k] + Z[(r - 12) * 4 + k] + Z[(r + 1) * 4 + k] + Z[(r - 1) * 4 + k] + zp + zm;
    const float pgs = (sum - s.BZ[(a * 8 + b) * 2 + hi] * dx2) * dev::kInv6;
    const float po = Z[r * 4 + k];
    s.PZ[r * 4 + k] = po + omega * (pgs - po);
}

// Copy descriptor q in [0, 58): source leaf (neighbour index), source slot offset, size in
// floats, destination offset in floats within Smem (P = 0, B = P + 1152).
struct CopyDesc {
    int nb, slot, count, dst, field;  // field 0 = p, 1 = div
};

__device__ __forceinline__ CopyDesc copy_desc(int q) {
    CopyDesc c;
    if (q < 8) {  // p interior plane a = q
        c = {nbi(0, 0, 0), q * 64, 64, prow(q, 0) * 8, 0};
    } else if (q < 10) {  // p -x face: planes x = 6, 7 of the -x leaf -> a = -2, -1
        const int a = q - 10;
        c = {nbi(-1, 0, 0), (a + 8) * 64, 64, prow(a, 0) * 8, 0};
    } else if (q < 12) {  // p +x face: planes x = 0, 1 -> a = 8, 9
        const int a = q - 2;
        c = {nbi(1, 0, 0), (a - 8) * 64, 64, prow(a, 0) * 8, 0};
    } else if (q < 20) {  // p -y face of plane a: rows y = 6, 7 -> b = -2, -1
        const int a = q - 12;
        c = {nbi(0, -1, 0), a * 64 + 48, 16, prow(a, -2) * 8, 0};
    } else if (q < 28) {  // p +y face of plane a: rows y = 0, 1 -> b = 8, 9
        const int a = q - 20;
        c = {nbi(0, 1, 0), a * 64, 16, prow(a, 8) * 8, 0};
    } else if (q < 32) {  // p xy-edge rows (a, b) in {-1, 8}^2
        const int a = (q & 2) ? 8 : -1, b = (q & 1) ? 8 : -1;
        c = {nbi(a < 0 ? -1 : 1, b < 0 ? -1 : 1, 0), (a & 7) * 64 + (b & 7) * 8, 8, prow(a, b) * 8, 0};
    } else if (q < 40) {  // div interior plane
        const int a = q - 32;
        c = {nbi(0, 0, 0), a * 64, 64, 1152 + brow(a, 0) * 8, 1};
    } else if (q == 40) {  // div -x face plane x = 7 -> a = -1
        c = {nbi(-1, 0, 0), 7 * 64, 64, 1152 + brow(-1, 0) * 8, 1};
    } else if (q == 41) {  // div +x face plane x = 0 -> a = 8
        c = {nbi(1, 0, 0), 0, 64, 1152 + brow(8, 0) * 8, 1};
    } else if (q < 50) {  // div -y face of plane a: row y = 7 -> b = -1
        const int a = q - 42;
        c = {nbi(0, -1, 0), a * 64 + 56, 8, 1152 + brow(a, -1) * 8, 1};
    } else {  // div +y face of plane a: row y = 0 -> b = 8
        const int a = q - 50;
        c = {nbi(0, 1, 0), a * 64, 8, 1152 + brow(a, 8) * 8, 1};
    }
    return c;
}

constexpr int kCopies = 58;

// Bit q set: copy q has no source (missing neighbour leaf, or p = 0) and its destination is
// zero-filled instead. Each warp computes the mask itself (two descriptors per lane).
__device__ __forceinline__ uint64_t missing_mask(const Smem& s, bool p_zero, int lane) {
    uint32_t lo = 0, hi = 0;
    {
        const CopyDesc c = copy_desc(lane);
        lo = __ballot_sync(0xffffffffu, (c.field == 0 && p_zero) || s.nb[c.nb] < 0);
    }
    {
        const int q = lane + 32;
        bool m = false;
        if (q < kCopies) {
            const CopyDesc c = copy_desc(q);
            m = (c.field == 0 && p_zero) || s.nb[c.nb] < 0;
        }
        hi = __ballot_sync(0xffffffffu, m);
    }
    return (uint64_t)lo | ((uint64_t)hi << 32);
}

template <int NT>
__global__ void __launch_bounds__(NT) rbgs_bulk_kernel(TopoView t, const float* __restrict__ div,
                                                        const float* __restrict__ p_in, float* __restrict__ p_out,
                                                        float dx2, float omega, const double* __restrict__ check,
                                                        double tol2, double* __restrict__ resid_out,
                                                        unsigned long long* __restrict__ counters) {
    __shared__ __align__(128) Smem s;
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int64_t leaf = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 27) s.nb[tid] = __ldg(t.nbr27 + leaf * 27 + tid);
    if (tid == 32) {
        ptx::mbar_init(&s.bar, 1);
        ptx::fence_barrier_init();
        if (counters != nullptr && leaf == 0) atomicAdd(counters, 1ull);
    }
    __syncthreads();

    float* base = s.P;  // P and B are adjacent: B = P + 1152 floats
    const uint64_t missing = missing_mask(s, p_in == nullptr, lane);
    if (warp == 0) {
        // Bytes the existing copies will deliver, then the copies themselves.
        uint32_t bytes = 0;
        for (int q = lane; q < kCopies; q += 32)
            if (!((missing >> q) & 1)) bytes += (uint32_t)copy_desc(q).count * 4u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (lane == 0) ptx::mbar_arrive_expect_tx(&s.bar, bytes);
        __syncwarp();
        for (int q = lane; q < kCopies; q += 32) {
            if ((missing >> q) & 1) continue;
            const CopyDesc c = copy_desc(q);
            const float* src = c.field == 0 ? p_in : div;
            ptx::bulk_g2s(base + c.dst, src + ((int64_t)s.nb[c.nb] << 9) + c.slot, (uint32_t)c.count * 4u, &s.bar);
        }
    } else {
        // The z-halo with plain loads, spread over the other warps:
        //   u in [0, 128):   p at z = -2, -1 / 8, 9 and div at z = -1 / 8 of interior row (a, b)
        //   u in [128, 192): p at z = -1 / 8 of an x/y ring row, from the edge leaves.
        for (int u = tid - 32; u < 192; u += NT - 32) {
            if (u < 128) {
                const int hi = u >> 6, row = u & 63, a = row >> 3, b = row & 7;
                const int l = s.nb[hi ? nbi(0, 0, 1) : nbi(0, 0, -1)];
                float2 pz = make_float2(0.f, 0.f);
                float dz = 0.f;
                if (l >= 0) {
                    const int64_t rs = ((int64_t)l << 9) + a * 64 + b * 8;
                    if (p_in != nullptr) pz = __ldg(reinterpret_cast<const float2*>(p_in + rs + (hi ? 0 : 6)));
                    dz = __ldg(div + rs + (hi ? 0 : 7));
                }
                float* z = &s.PZ[prow(a, b) * 4 + (hi ? 2 : 0)];
                z[0] = pz.x;
                z[1] = pz.y;
                s.BZ[(a * 8 + b) * 2 + hi] = dz;
            } else {
                const int v = u - 128, side = v >> 4, hi = (v >> 3) & 1, k = v & 7;
                int a, b, la, lb;
                if (side == 0) a = -1, b = k, la = -1, lb = 0;
                else if (side == 1) a = 8, b = k, la = 1, lb = 0;
                else if (side == 2) a = k, b = -1, la = 0, lb = -1;
                else a = k, b = 8, la = 0, lb = 1;
                const int l = s.nb[nbi(la, lb, hi ? 1 : -1)];
                float val = 0.f;
                if (l >= 0 && p_in != nullptr) val = __ldg(p_in + ((int64_t)l << 9) + (a & 7) * 64 + (b & 7) * 8 + (hi ? 0 : 7));
                s.PZ[prow(a, b) * 4 + (hi ? 2 : 1)] = val;
            }
        }
        // Zero-fill the destinations of missing copies (none for a leaf deep inside the domain).
        uint64_t m = missing;
        while (m) {
            const int q = __ffsll((long long)m) - 1;
            m &= m - 1;
            const CopyDesc c = copy_desc(q);
            for (int i = tid - 32; i < c.count; i += NT - 32) base[c.dst + i] = 0.f;
        }
    }
    __syncthreads();
    if (!ptx::mbar_wait_bounded(&s.bar, 0, kMaxPolls)) {
        // The copies did not land in time: flag it, give them a second bounded wait so that
        // no copy is still writing when the CTA's shared memory is released, and leave p_out
        // untouched for this leaf.
        if (tid == 0 && counters != nullptr) atomicExch(counters + 1, 1ull);
        (void)ptx::mbar_wait_bounded(&s.bar, 0, kMaxPolls);
        return;
    }

    if (resid_out != nullptr) {
        const double h2 = (double)dx2;
        double r2 = 0.0, b2 = 0.0;
        for (int n = tid; n < 512; n += NT) {
            const int a = n >> 6, b = (n >> 3) & 7, d = n & 7;
            const double lap = (double)pv(s, a + 1, b, d) + (double)pv(s, a - 1, b, d) + (double)pv(s, a, b + 1, d) +
                               (double)pv(s, a, b - 1, d) + (double)pv(s, a, b, d + 1) + (double)pv(s, a, b, d - 1) -
                               6.0 * (double)pv(s, a, b, d);
            const double bb = (double)bv(s, a, b, d) * h2;
            r2 += (bb - lap) * (bb - lap);
            b2 += bb * bb;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        if (lane == 0) s.red[0][warp] = r2, s.red[1][warp] = b2;
        __syncthreads();
        if (tid < 32) {
            r2 = tid < NT / 32 ? s.red[0][tid] : 0.0;
            b2 = tid < NT / 32 ? s.red[1][tid] : 0.0;
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

    // Red (colour 0): 256 voxels of the leaf, then 32 per face of the ring whose leaf exists.
    // Leaf origins are multiples of 8, so a voxel's colour is the parity of a + b + d.
    for (int r = tid; r < 448; r += NT) {
        if (r < 256) {
            const int row = r >> 2, a = row >> 3, b = row & 7;
            relax_row(s, prow(a, b), brow(a, b), 2 * (r & 3) + ((a + b) & 1), dx2, omega);
        } else {
            const int f = (r - 256) >> 5, k = (r - 256) & 31, u = k >> 2;
            const int fixed = (f & 1) ? 8 : -1;
            const int v = 2 * (k & 3) + ((u + fixed) & 1);
            if (f < 2) {
                if (s.nb[nbi(f ? 1 : -1, 0, 0)] >= 0) relax_row(s, prow(fixed, u), brow(fixed, u), v, dx2, omega);
            } else if (f < 4) {
                if (s.nb[nbi(0, (f & 1) ? 1 : -1, 0)] >= 0) relax_row(s, prow(u, fixed), brow(u, fixed), v, dx2, omega);
            } else {
                if (s.nb[nbi(0, 0, (f & 1) ? 1 : -1)] >= 0) relax_zring(s, u, v, f & 1, dx2, omega);
            }
        }
    }
    __syncthreads();
    for (int r = tid; r < 256; r += NT) {  // Black (colour 1): 256 voxels of the leaf.
        const int row = r >> 2, a = row >> 3, b = row & 7;
        relax_row(s, prow(a, b), brow(a, b), 2 * (r & 3) + ((a + b + 1) & 1), dx2, omega);
    }
    __syncthreads();
    for (int q = tid; q < 128; q += NT) {
        const int a = q >> 4, o = (q & 15) * 4;
        const float4 v = *reinterpret_cast<const float4*>(&s.P[prow(a, 0) * 8 + o]);
        *reinterpret_cast<float4*>(p_out + (leaf << 9) + a * 64 + o) = v;
    }
}

}  // namespace

bool rbgs_bulk_eligible(const float* div, const float* p_in, const float* p_out) {
    const auto aligned = [](const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    return aligned(div) && aligned(p_in) && aligned(p_out);
}

void launch_rbgs_bulk(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                      const double* check, double tol2, double* resid_out) {
    if (c.rbgs_threads == 128)
        rbgs_bulk_kernel<128><<<(unsigned)c.topo.num_leaves, 128, 0, c.stream>>>(c.topo.view, div, p_in, p_out, c.dx * c.dx,
                                                                                  omega, check, tol2, resid_out, c.counters);
    else
        rbgs_bulk_kernel<256><<<(unsigned)c.topo.num_leaves, 256, 0, c.stream>>>(c.topo.view, div, p_in, p_out, c.dx * c.dx,
                                                                                  omega, check, tol2, resid_out, c.counters);
    HNS_LAUNCHED();
}

}  // namespace hns
