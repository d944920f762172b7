// The red-black SOR iteration, staged with bulk async copies and relaxed row by row.
//
// One 128-thread CTA per 8^3 leaf performs one full iteration of redBlackGaussSeidelUpdate
// (src/Cuda/Kernel.cu:459-489) -- red on the leaf and its one-voxel face ring, then black on
// the leaf -- from p_in to p_out, reading p with a two-voxel halo and the right-hand side
// with a one-voxel halo, as rbgs_iteration_kernel in hns_kernels.cu does (same arithmetic,
// same results to the bit). How the stencil reaches shared memory and is computed:
//
//   * Shared memory holds z-rows of 8 values. A leaf's slot order is x-major
//     (x*64 + y*8 + z), so every x-plane of a leaf (64 values), every pair of y-rows of a
//     plane (16 values) and every single row (8 values) is contiguous in HBM and lands
//     contiguously in the row layout: 58 pieces (8 interior planes, x-face planes, y-face
//     rows, xy-edge rows of p and of the right-hand side) are fetched by cp.async.bulk,
//     issued by one warp -- lane a issues the six pieces of plane a -- and counted on one
//     mbarrier. A piece whose leaf does not exist is zero-filled by the same lane.
//   * The z-halo (values at z = -2, -1, 8, 9 of a row) is one or two values per 32-byte
//     row in HBM; it is fetched with plain loads into separate arrays while the bulk
//     copies are in flight.
//   * Voxels are relaxed one per lane in warp tasks of 32 whose shared-memory reads hit 32
//     different banks (relax_task). Red: the leaf's 256, the x/y ring's 128 and the z
//     ring's 64; black: the leaf's 256.
//
// T is the storage type of p and the right-hand side (float, or __half for the inner solve
// of the mixed-precision refinement); arithmetic is FP32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "hns_internal.cuh"
#include "hns_ptx.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

constexpr int NT = 128;
// Bounded mbarrier wait: at most kMaxPolls polls of at most kSuspendNs each -- far above
// any real copy latency (microseconds), and about 1 s when every poll sleeps its full hint.
constexpr uint32_t kSuspendNs = 20000;
constexpr uint32_t kMaxPolls = 50000;

// Neighbour-table index of the leaf at offset (dx, dy, dz) in {-1,0,1}^3.
__host__ __device__ constexpr int nbi(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }

template <typename T>
struct Smem {
    T P[12 * 12 * 8];   // p rows: (a+2, b+2) for a, b in [-2, 9], z in [0, 8)
    T B[10 * 10 * 8];   // right-hand-side rows: (a+1, b+1) for a, b in [-1, 8]
    T PZ[12 * 12 * 4];  // p at z = -2, -1, 8, 9 of row (a+2, b+2)
    T BZ[8 * 8 * 2];    // right-hand side at z = -1, 8 of leaf row (a, b)
    double red[2][NT / 32];
    uint64_t bar;
    int nb[27];
    int wait_ok;
};

__device__ __forceinline__ int prow(int a, int b) { return (a + 2) * 12 + (b + 2); }
__device__ __forceinline__ int brow(int a, int b) { return (a + 1) * 10 + (b + 1); }

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

// One SOR update at (a, b, d), d in [0, 8), of a row r = prow(a, b) whose x/y neighbour
// rows are staged (the leaf's rows and the x/y ring rows): neighbour rows r +- 12 (x) and
// r +- 1 (y), z-halo PZ[4r+1] (z = -1) and PZ[4r+2] (z = 8), right-hand-side row rb. The
// six-neighbour sum is in the reference's order (x+, x-, y+, y-, z+, z-).
template <typename T>
__device__ __forceinline__ void relax_cell(Smem<T>& s, int r, int rb, int d, float dx2, float omega) {
    const T* P = s.P;
    const int c = r * 8 + d;
    const float zp = d < 7 ? to_f(P[c + 1]) : to_f(s.PZ[r * 4 + 2]);
    const float zm = d > 0 ? to_f(P[c - 1]) : to_f(s.PZ[r * 4 + 1]);
    const float sum = to_f(P[c + 96]) + to_f(P[c - 96]) + to_f(P[c + 8]) + to_f(P[c - 8]) + zp + zm;
    const float pgs = (sum - to_f(s.B[rb * 8 + d]) * dx2) * dev::kInv6;
    const float po = to_f(P[c]);
    s.P[c] = from_f<T>(po + omega * (pgs - po));
}

// The same update at a z-ring voxel (a, b, -1) (hi = 0) or (a, b, 8) (hi = 1), a, b in [0, 8):
// the voxel and its x/y neighbours live in the z-halo arrays.
template <typename T>
__device__ __forceinline__ void relax_zring(Smem<T>& s, int a, int b, int hi, float dx2, float omega) {
    const int r = prow(a, b), k = hi ? 2 : 1;
    const T* Z = s.PZ;
    const float zp = hi ? to_f(Z[r * 4 + 3]) : to_f(s.P[r * 8 + 0]);
    const float zm = hi ? to_f(s.P[r * 8 + 7]) : to_f(Z[r * 4 + 0]);
    const float sum = to_f(Z[(r + 12) * 4 + k]) + to_f(Z[(r - 12) * 4 + k]) + to_f(Z[(r + 1) * 4 + k]) +
                      to_f(Z[(r - 1) * 4 + k]) + zp + zm;
    const float pgs = (sum - to_f(s.BZ[(a * 8 + b) * 2 + hi]) * dx2) * dev::kInv6;
    const float po = to_f(Z[r * 4 + k]);
    s.PZ[r * 4 + k] = from_f<T>(po + omega * (pgs - po));
}

// The cells of one warp task, one per lane, chosen so that the 32 lanes' shared-memory
// reads fall in 32 different banks: a task covers 4 consecutive y-rows of two x-rows 12 rows
// apart (the same bank base) whose voxels of the current colour have opposite parity in d
// (odd and even banks), 4 voxels per row. Tasks 0-7: the leaf's rows; red only: 8-9 the
// x-ring rows, 10-11 the y-ring rows, 12-13 the z-ring voxels.
template <typename T>
__device__ __forceinline__ void relax_task(Smem<T>& s, int task, int lane, int colour, float dx2, float omega) {
    const int k = lane & 3, q = (lane >> 2) & 3, h = (lane >> 4) & 1;
    if (task < 8) {  // leaf rows: a = 2 (task >> 1) + h, b = 4 (task & 1) + q
        const int a = 2 * (task >> 1) + h, b = 4 * (task & 1) + q;
        relax_cell(s, prow(a, b), brow(a, b), 2 * k + (((a + b) & 1) ^ colour), dx2, omega);
    } else if (task < 10) {  // x-ring rows: a = -1 or 8 (by h), b = 4 (task - 8) + q
        const int a = h ? 8 : -1, b = 4 * (task - 8) + q;
        if (s.nb[nbi(h ? 1 : -1, 0, 0)] >= 0) relax_cell(s, prow(a, b), brow(a, b), 2 * k + ((a + b) & 1), dx2, omega);
    } else if (task < 12) {  // y-ring rows: b = -1 or 8 (by h), a = 4 (task - 10) + q
        const int a = 4 * (task - 10) + q, b = h ? 8 : -1;
        if (s.nb[nbi(0, h ? 1 : -1, 0)] >= 0) relax_cell(s, prow(a, b), brow(a, b), 2 * k + ((a + b) & 1), dx2, omega);
    } else {  // z-ring: row (a, b) has its red voxel at z = 8 if a+b is even, else at z = -1
        const int row = (task - 12) * 32 + lane, a = row >> 3, b = row & 7, hi = ((a + b) & 1) == 0;
        if (s.nb[nbi(0, 0, hi ? 1 : -1)] >= 0) relax_zring(s, a, b, hi, dx2, omega);
    }
}

// Value of p at local (a, b, d), d in [-2, 9] (residual evaluation).
template <typename T>
__device__ __forceinline__ float pv(const Smem<T>& s, int a, int b, int d) {
    const int r = prow(a, b);
    if ((unsigned)d < 8u) return to_f(s.P[r * 8 + d]);
    return to_f(s.PZ[r * 4 + (d < 0 ? d + 2 : d - 6)]);
}

template <typename T>
__device__ __forceinline__ float bv(const Smem<T>& s, int a, int b, int d) {
    if ((unsigned)d < 8u) return to_f(s.B[brow(a, b) * 8 + d]);
    return to_f(s.BZ[(a * 8 + b) * 2 + (d < 0 ? 0 : 1)]);
}

// One staged piece: `count` values of leaf `l` from slot offset `slot` to shared `dst`,
// fetched by a bulk copy, or zeros when the leaf (or the array) does not exist.
template <typename T>
struct Piece {
    const T* src;
    int l, slot, count;
    T* dst;
};

template <typename T>
__device__ __forceinline__ void piece_issue(const Piece<T>& pc, uint64_t* bar) {
    if (pc.src != nullptr && pc.l >= 0) {
        ptx::bulk_g2s(pc.dst, pc.src + ((int64_t)pc.l << 9) + pc.slot, (uint32_t)(pc.count * sizeof(T)), bar);
    } else {
        for (int i = 0; i < pc.count; ++i) pc.dst[i] = from_f<T>(0.f);
    }
}

template <typename T>
__device__ __forceinline__ uint32_t piece_bytes(const Piece<T>& pc) {
    return (pc.src != nullptr && pc.l >= 0) ? (uint32_t)(pc.count * sizeof(T)) : 0u;
}

template <typename T>
__global__ void __launch_bounds__(NT) rbgs_bulk_kernel(TopoView t, const T* __restrict__ rhs,
                                                        const T* __restrict__ p_in, T* __restrict__ p_out,
                                                        float dx2, float omega, const double* __restrict__ check,
                                                        double tol2, double* __restrict__ resid_out,
                                                        unsigned long long* __restrict__ counters) {
    __shared__ __align__(128) Smem<T> s;
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

    if (warp == 0) {
        // Lanes 0-7: plane a = lane -- p and rhs interior planes, p y-face row pairs
        // (y = 6,7 of the -y leaf; y = 0,1 of the +y leaf), rhs y-face rows.
        // Lanes 8-11: p x-face planes; 12-13: rhs x-face planes; 14-17: p xy-edge rows.
        Piece<T> pcs[6];
        int np = 0;
        if (lane < 8) {
            const int a = lane, lmy = s.nb[nbi(0, -1, 0)], lpy = s.nb[nbi(0, 1, 0)];
            pcs[0] = {p_in, (int)leaf, a * 64, 64, &s.P[prow(a, 0) * 8]};
            pcs[1] = {rhs, (int)leaf, a * 64, 64, &s.B[brow(a, 0) * 8]};
            pcs[2] = {p_in, lmy, a * 64 + 48, 16, &s.P[prow(a, -2) * 8]};
            pcs[3] = {p_in, lpy, a * 64, 16, &s.P[prow(a, 8) * 8]};
            pcs[4] = {rhs, lmy, a * 64 + 56, 8, &s.B[brow(a, -1) * 8]};
            pcs[5] = {rhs, lpy, a * 64, 8, &s.B[brow(a, 8) * 8]};
            np = 6;
        } else if (lane < 12) {
            const int q = lane - 8, a = (q < 2) ? q - 2 : q + 6;  // -2, -1, 8, 9
            const int l = s.nb[nbi(a < 0 ? -1 : 1, 0, 0)];
            pcs[0] = {p_in, l, (a & 7) * 64, 64, &s.P[prow(a, 0) * 8]};
            np = 1;
        } else if (lane < 14) {
            const int a = lane == 12 ? -1 : 8;
            pcs[0] = {rhs, s.nb[nbi(a < 0 ? -1 : 1, 0, 0)], (a & 7) * 64, 64, &s.B[brow(a, 0) * 8]};
            np = 1;
        } else if (lane < 18) {
            const int q = lane - 14, a = (q & 2) ? 8 : -1, b = (q & 1) ? 8 : -1;
            pcs[0] = {p_in, s.nb[nbi(a < 0 ? -1 : 1, b < 0 ? -1 : 1, 0)], (a & 7) * 64 + (b & 7) * 8, 8, &s.P[prow(a, b) * 8]};
            np = 1;
        }
        uint32_t bytes = 0;
        for (int i = 0; i < np; ++i) bytes += piece_bytes(pcs[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (lane == 0) ptx::mbar_arrive_expect_tx(&s.bar, bytes);
        __syncwarp();
        for (int i = 0; i < np; ++i) piece_issue(pcs[i], &s.bar);
    }
    // The z-halo with plain loads, one task per thread (warp 0 after issuing its copies):
    //   tid in [0, 128):  p at z = -2,-1 (tid < 64, from the -z leaf) or z = 8,9 (from the +z
    //                     leaf) and rhs at z = -1 / 8 of leaf row (a, b) = (row >> 3, row & 7)
    //   tid in [64, 128): also p at z = -1 / 8 of an x/y ring row, from the edge leaves.
    {
        const int hi = tid >> 6, row = tid & 63, a = row >> 3, b = row & 7;
        const int l = s.nb[hi ? nbi(0, 0, 1) : nbi(0, 0, -1)];
        T pz0 = from_f<T>(0.f), pz1 = from_f<T>(0.f), dz = from_f<T>(0.f);
        if (l >= 0) {
            const int64_t rs = ((int64_t)l << 9) + a * 64 + b * 8 + (hi ? 0 : 6);
            if (p_in != nullptr) pz0 = p_in[rs], pz1 = p_in[rs + 1];
            dz = rhs[rs + (hi ? 0 : 1)];
        }
        T* z = &s.PZ[prow(a, b) * 4 + (hi ? 2 : 0)];
        z[0] = pz0;
        z[1] = pz1;
        s.BZ[(a * 8 + b) * 2 + hi] = dz;
    }
    if (tid >= 64) {
        const int v = tid - 64, side = v >> 4, zhi = (v >> 3) & 1, k = v & 7;
        int a, b, la, lb;
        if (side == 0) a = -1, b = k, la = -1, lb = 0;
        else if (side == 1) a = 8, b = k, la = 1, lb = 0;
        else if (side == 2) a = k, b = -1, la = 0, lb = -1;
        else a = k, b = 8, la = 0, lb = 1;
        const int l = s.nb[nbi(la, lb, zhi ? 1 : -1)];
        T val = from_f<T>(0.f);
        if (l >= 0 && p_in != nullptr) val = p_in[((int64_t)l << 9) + (a & 7) * 64 + (b & 7) * 8 + (zhi ? 0 : 7)];
        s.PZ[prow(a, b) * 4 + (zhi ? 2 : 1)] = val;
    }
    // One thread waits for the copies (sleeping between polls); the others wait at the CTA
    // barrier, which costs no issue slots.
    if (tid == 0) {
        s.wait_ok = ptx::mbar_wait_bounded_sleep(&s.bar, 0, kMaxPolls, kSuspendNs) ? 1 : 0;
        if (!s.wait_ok) {
            // The copies did not land in time: flag it and give them a second bounded wait so
            // that no copy is still writing when the CTA's shared memory is released.
            if (counters != nullptr) atomicExch(counters + 1, 1ull);
            (void)ptx::mbar_wait_bounded_sleep(&s.bar, 0, kMaxPolls, kSuspendNs);
        }
    }
    __syncthreads();
    if (!s.wait_ok) return;  // leave p_out untouched for this leaf

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

    // Red (colour 0), then black (colour 1): leaf origins are multiples of 8, so a voxel's
    // colour is the parity of its local a + b + d.
    for (int task = warp; task < 14; task += NT / 32) relax_task(s, task, lane, 0, dx2, omega);
    __syncthreads();
    for (int task = warp; task < 8; task += NT / 32) relax_task(s, task, lane, 1, dx2, omega);
    __syncthreads();
    constexpr int kVec = 16 / sizeof(T);  // values per 16-byte store
    for (int q = tid; q < 512 / kVec; q += NT) {
        const int a = (q * kVec) >> 6, o = (q * kVec) & 63;
        *reinterpret_cast<uint4*>(p_out + (leaf << 9) + a * 64 + o) = *reinterpret_cast<const uint4*>(&s.P[prow(a, 0) * 8 + o]);
    }
}

template <typename T>
bool aligned16(const T* p) {
    return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

}  // namespace

bool rbgs_bulk_eligible(const float* div, const float* p_in, const float* p_out) {
    return aligned16(div) && aligned16(p_in) && aligned16(p_out);
}

void launch_rbgs_bulk(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                      const double* check, double tol2, double* resid_out) {
    rbgs_bulk_kernel<float><<<(unsigned)c.topo.num_leaves, NT, 0, c.stream>>>(c.topo.view, div, p_in, p_out, c.dx * c.dx,
                                                                              omega, check, tol2, resid_out, c.counters);
    HNS_LAUNCHED();
}

void launch_rbgs_bulk_unit(const Context& c, const float* rhs, const float* e_in, float* e_out, float omega,
                           const double* check, double tol2) {
    if (!aligned16(rhs) || !aligned16(e_in) || !aligned16(e_out)) fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be 16-byte aligned");
    rbgs_bulk_kernel<float><<<(unsigned)c.topo.num_leaves, NT, 0, c.stream>>>(c.topo.view, rhs, e_in, e_out, 1.0f, omega, check,
                                                                              tol2, nullptr, c.counters);
    HNS_LAUNCHED();
}

void launch_rbgs_bulk_half(const Context& c, const void* rhs, const void* e_in, void* e_out, float omega,
                           const double* check, double tol2) {
    const __half* r = static_cast<const __half*>(rhs);
    const __half* ei = static_cast<const __half*>(e_in);
    __half* eo = static_cast<__half*>(e_out);
    if (!aligned16(r) || !aligned16(ei) || !aligned16(eo)) fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be 16-byte aligned");
    rbgs_bulk_kernel<__half><<<(unsigned)c.topo.num_leaves, NT, 0, c.stream>>>(c.topo.view, r, ei, eo, 1.0f, omega, check, tol2,
                                                                               nullptr, c.counters);
    HNS_LAUNCHED();
}

}  // namespace hns
