// The red-black SOR half-sweep on colour-split FP16 leaves: the inner solve of the
// mixed-precision refinement (L e = r with unit spacing, e and r in FP16, FP32 arithmetic), one
// launch per colour, in place.
//
// Layout. The inner solve's arrays belong to the solver, so their layout is free. Each leaf
// stores its 256 red values (colour (x + y + z) & 1 = 0) and then its 256 black values. Within
// a colour, entry 4 R + j is the row (local x = a, y = b) at position
// R = 32 ((a + b) & 1) + 4 a + (b >> 1), at the j-th z of that colour in the row:
// z = 2 j + ((a + b + colour) & 1). A colour of a row is 8 contiguous bytes, and the 32 rows of
// one parity of a + b are 256 contiguous bytes: one warp's load.
//
// Neighbours of voxel (a, b, z = 2 j + p) of colour c: its x and y neighbours are entry j of
// the other colour in rows (a -+ 1, b) and (a, b -+ 1) (in the neighbour leaf across a face,
// rows wrapped mod 8), all of the other parity of a + b; its z neighbours are entries of the
// other colour of its own row: j - 1 and j for p = 0, j and j + 1 for p = 1, where entry -1 is
// the -z leaf's entry 3 of that row and entry 4 the +z leaf's entry 0. A missing leaf reads 0
// (the reference's p = 0 outside the domain).
//
// Work: a thread relaxes the four voxels of one colour of a row, in four leaves, from eight
// 8-byte loads per leaf (the row's two colours, its right-hand side, the four neighbour rows)
// and one of 2 bytes, and one 8-byte store. A half-sweep reads both colours of e and the
// colour's right-hand side and writes the colour in place: about 3 bytes per voxel from DRAM,
// with no staging, no halo copies and no second buffer of e. The update of each voxel is
// relax16::relax1, the arithmetic of every other FP16 inner kernel, so all layouts give the
// same values to the bit (the tests compare them). Sweeps follow redBlackGaussSeidelUpdate
// (src/Cuda/Kernel.cu:459-489): red, then black, per iteration.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "hns_internal.cuh"
#include "hns_relax16.cuh"

namespace hns {
namespace {

using namespace relax16;

// Measured on a 45,198-leaf grid (us per half-sweep): 4 x 2 (256 threads) 18.3, 4 x 3 17.4,
// 2 x 3 17.1, 1 x 5 16.8, 2 x 4 16.7, 2 x 6 17.4, 1 x 1 22.2: more leaves per thread keep more
// loads in flight, and small blocks leave a shorter tail to the last wave.
// Register limit: 80 registers give 6 CTAs per SM; 64 registers (8 per SM) measured 19.8 us with
// four leaves per thread (spills), 16.2 with three, 17.5 with two: no gain over 6 x 4 (16.1).
// A thread per row quad (the four same-parity rows at one x: 16-byte loads, 15 loads for 16
// updates instead of 36, same values) measured 18.6 us at 6 CTAs per SM and 16.8 at 8: fewer
// instructions, but fewer bytes in flight, and the kernel is bound by memory latency.
constexpr int kLeavesPerBlock = 2;   // leaves whose rows one block's threads cover
constexpr int kLeavesPerThread = 4;  // leaves a thread relaxes its row in
constexpr int kThreads = 64 * kLeavesPerBlock;
constexpr int kShortGridCtasPerSm = 6;  // the register limit at 80 registers and 128 threads
constexpr int kHalfCtasPerSm = 6;       // the half-sweep kernel's launch bound

// nbr27 indices of the six face neighbours: (dx+1)*9 + (dy+1)*3 + (dz+1).
constexpr int kNbXp = 22, kNbXm = 4, kNbYp = 16, kNbYm = 10, kNbZp = 14, kNbZm = 12;

__device__ __forceinline__ uint2 ld8(const __half* p) { return __ldg(reinterpret_cast<const uint2*>(p)); }
// Loads that other threads of this launch may write: the colour being updated is only read by
// the thread that writes it, so plain (non-.nc) loads of it are enough; the other colour is
// read-only during the launch.
__device__ __forceinline__ uint2 ld8_rw(const __half* p) { return *reinterpret_cast<const uint2*>(p); }

__device__ __forceinline__ uint32_t half_at(uint2 v, int j) {
    const uint32_t w = (j & 2) ? v.y : v.x;
    return (j & 1) ? (w >> 16) : (w & 0xFFFFu);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __half2 r = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&r);
}

// Face-neighbour table of the half-sweep: per leaf {+x, -x, +y, -y, +z, -z, the leaf, 0}, a
// missing neighbour replaced by the zero leaf (index L, just past the last leaf of e, which the
// sweeps read and never write), so that no load needs a test.
__global__ void split_face_table_kernel(TopoView t, int4* __restrict__ nb8) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= t.num_leaves) return;
    const int* nb = t.nbr27 + l * 27;
    const int L = (int)t.num_leaves;
    auto f = [&](int k) { const int v = __ldg(nb + k); return v < 0 ? L : v; };
    nb8[2 * l] = make_int4(f(kNbXp), f(kNbXm), f(kNbYp), f(kNbYm));
    nb8[2 * l + 1] = make_int4(f(kNbZp), f(kNbZm), (int)l, 0);
}

// One row's update for z parity P of its colour (P = 0: z = 0, 2, 4, 6): z neighbours are
// entries j - 1 and j (P = 0) or j and j + 1 (P = 1) of the row's other colour K, with ZC the
// entry across the z face.
template <int P>
__device__ __forceinline__ uint2 relax_row(uint2 XP, uint2 XM, uint2 YP, uint2 YM, uint2 K, uint32_t ZC, uint2 B,
                                           uint2 C, float omega) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t zm = P ? half_at(K, j) : (j > 0 ? half_at(K, j - 1) : ZC);
        const uint32_t zp = P ? (j < 3 ? half_at(K, j + 1) : ZC) : half_at(K, j);
        v[j] = relax1(half_at(XP, j), half_at(XM, j), half_at(YP, j), half_at(YM, j), zp, zm, half_at(B, j), half_at(C, j),
                      omega);
    }
    return make_uint2(pack2(v[0], v[1]), pack2(v[2], v[3]));
}

// One CTA pass of a half-sweep: relax the rows of colour `colour` in leaf group g (the
// kLeavesPerBlock * kLeavesPerThread leaves from g * kLeavesPerGroup).
//
// kZero: e = 0 before this (red) half-sweep, the first of a solve: every neighbour and old
// value is 0, nothing of e is read, and the row's black entries are written as 0.
// kShared: other CTAs of the same launch write e (the persistent solve): every load of e takes
// the coherent path; otherwise the colour not being updated is read-only during the launch and
// goes through the read-only cache. kPdl: wait for the preceding launch (griddepcontrol.wait)
// before the first load of e.
//
// Warp w of a leaf takes the 32 rows of parity w of a + b, lane l the row at R = 32 w + l
// (a = l / 4, b = 2 (l % 4) + ((a + w) & 1)), so the z parity of the colour is uniform in a warp
// and the z neighbours need no selects. A thread relaxes its row in kLeavesPerThread leaves
// (kLeavesPerBlock apart), issuing every load before any arithmetic: the kernel is bound by
// memory latency, and this multiplies the bytes each thread has in flight. Loads are
// unconditional: a row on a leaf face reads the neighbour leaf's row, a missing neighbour the
// zero leaf. Offsets are 32-bit element counts (fewer than 2^22 leaves).
constexpr int kLeavesPerGroup = kLeavesPerBlock * kLeavesPerThread;

template <bool kZero, bool kShared, bool kPdl, typename Mid>
__device__ __forceinline__ void relax_group(const int* __restrict__ nb8, const __half* __restrict__ rhs, __half* e,
                                            int num_leaves, int g, int colour, float omega, Mid&& mid) {
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) & 1;
    const int a = lane >> 2, b = 2 * (lane & 3) + ((a + w) & 1);
    const int p = (w + colour) & 1;  // z parity of this colour in the warp's rows
    const uint32_t rowc = ((uint32_t)colour << 8) | (uint32_t)(4 * (32 * w + lane));  // own entries within a leaf
    auto lde = [](const __half* q) { return kShared ? ld8_rw(q) : ld8(q); };
    const int leaf0 = g * kLeavesPerGroup + (int)(threadIdx.x >> 6);
    uint32_t own[kLeavesPerThread];
    bool live[kLeavesPerThread];
#pragma unroll
    for (int k = 0; k < kLeavesPerThread; ++k) {
        const int leaf = leaf0 + k * kLeavesPerBlock;
        live[k] = leaf < num_leaves;
        own[k] = ((uint32_t)(live[k] ? leaf : 0) << 9) | rowc;  // a dead slot reads leaf 0 and stores nothing
    }
    uint2 B[kLeavesPerThread], out[kLeavesPerThread];
#pragma unroll
    for (int k = 0; k < kLeavesPerThread; ++k) B[k] = ld8(rhs + own[k]);
    if constexpr (kZero) {
        mid();
#pragma unroll
        for (int k = 0; k < kLeavesPerThread; ++k) {
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = relax1(0u, 0u, 0u, 0u, 0u, 0u, half_at(B[k], j), 0u, omega);
            out[k] = make_uint2(pack2(v[0], v[1]), pack2(v[2], v[3]));
            if (live[k]) *reinterpret_cast<uint2*>(e + (own[k] ^ 256u)) = make_uint2(0u, 0u);
        }
    } else {
        // Row (a', b') of the other parity in the other colour of leaf n.
        const uint32_t co = ((uint32_t)(colour ^ 1) << 8) | (uint32_t)(128 * (w ^ 1));
        auto row = [&](uint32_t n, int a2, int b2) { return (n << 9) | co | (uint32_t)(16 * a2 + 4 * (b2 >> 1)); };
        const int sx = a == 7 ? 0 : a == 0 ? 1 : 6, sy = b == 7 ? 2 : b == 0 ? 3 : 6, sz = 5 - p;
        uint32_t nx[kLeavesPerThread], ny[kLeavesPerThread], nz[kLeavesPerThread];
#pragma unroll
        for (int k = 0; k < kLeavesPerThread; ++k) {
            const int* nb = nb8 + 8 * (own[k] >> 9);
            nx[k] = (uint32_t)__ldg(nb + sx);
            ny[k] = (uint32_t)__ldg(nb + sy);
            nz[k] = (uint32_t)__ldg(nb + sz);  // -z leaf for p = 0, +z for p = 1
        }
        // e is written by the preceding half-sweep: wait until it has finished (a no-op for a
        // launch without the programmatic-serialization attribute).
        if constexpr (kPdl) asm volatile("griddepcontrol.wait;" ::: "memory");
        uint2 C[kLeavesPerThread], K[kLeavesPerThread], XP[kLeavesPerThread], XM[kLeavesPerThread],
            YP[kLeavesPerThread], YM[kLeavesPerThread];
        uint32_t ZC[kLeavesPerThread];
#pragma unroll
        for (int k = 0; k < kLeavesPerThread; ++k) {
            C[k] = ld8_rw(e + own[k]);
            K[k] = lde(e + (own[k] ^ 256u));
        }
#pragma unroll
        for (int k = 0; k < kLeavesPerThread; ++k) {
            const uint32_t lf = own[k] >> 9;
            XP[k] = lde(e + row(a == 7 ? nx[k] : lf, (a + 1) & 7, b));
            XM[k] = lde(e + row(a == 0 ? nx[k] : lf, (a - 1) & 7, b));
            YP[k] = lde(e + row(b == 7 ? ny[k] : lf, a, (b + 1) & 7));
            YM[k] = lde(e + row(b == 0 ? ny[k] : lf, a, (b - 1) & 7));
            const __half* zq = e + ((nz[k] << 9) | ((own[k] ^ 256u) & 511u)) + 3u * (uint32_t)(p ^ 1);
            ZC[k] = kShared ? (uint32_t)*reinterpret_cast<const unsigned short*>(zq) : (uint32_t)__half_as_ushort(__ldg(zq));
        }
        mid();  // every load of the pass is in flight
#pragma unroll
        for (int k = 0; k < kLeavesPerThread; ++k)
            out[k] = p ? relax_row<1>(XP[k], XM[k], YP[k], YM[k], K[k], ZC[k], B[k], C[k], omega)
                       : relax_row<0>(XP[k], XM[k], YP[k], YM[k], K[k], ZC[k], B[k], C[k], omega);
    }
#pragma unroll
    for (int k = 0; k < kLeavesPerThread; ++k)
        if (live[k]) *reinterpret_cast<uint2*>(e + own[k]) = out[k];
}

// One half-sweep per launch. Leaf groups: one per CTA in a full grid; a short grid loops. Within
// a launch a thread reads and writes only its own rows of the launch's colour and only reads the
// other colour, so the passes of a CTA are independent.
template <bool kZero>
__global__ void __launch_bounds__(kThreads, kHalfCtasPerSm) rbgs_split_half_kernel(const int* __restrict__ nb8,
                                                                    const __half* __restrict__ rhs, __half* e,
                                                                    int num_leaves, int colour, float omega,
                                                                    const double* __restrict__ check, double tol2,
                                                                    unsigned long long* __restrict__ counters) {
    if (check != nullptr && check[0] <= tol2 * check[1]) return;  // the refinement has converged
    if (counters != nullptr && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(counters, 1ull);  // half-sweeps that ran
    // The next half-sweep may be scheduled as soon as every block of this one has started: its
    // blocks take the SM slots this launch's last wave frees and load what no sweep writes
    // before they wait for this launch to finish.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int groups = (num_leaves + kLeavesPerGroup - 1) / kLeavesPerGroup;
    for (int g = blockIdx.x; g < groups; g += gridDim.x)
        relax_group<kZero, false, true>(nb8, rhs, e, num_leaves, g, colour, omega, [] {});
}

// ---- FP32 ---------------------------------------------------------------------------------
// The same half-sweep on FP32 values, the reference's precision: the colour-split layout of e
// with rows of 4 floats (16 bytes), the right-hand side the divergence in the same layout, and
// the update of redBlackGaussSeidelUpdate as the staged FP32 kernel computes it:
// pgs = (x+ + x- + y+ + y- + z+ + z- - div dx^2) * 0.166666667f, p = p + omega (pgs - p), so the
// two kernels give the same values. Rows of 16 bytes hold twice the registers of the FP16 rows:
// two leaves per thread.
constexpr int kF32LeavesPerBlock = 2;
constexpr int kF32LeavesPerThread = 2;
constexpr int kF32Threads = 64 * kF32LeavesPerBlock;
constexpr int kF32ShortGridCtasPerSm = 8;

__device__ __forceinline__ float4 ldf4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 ldf4_rw(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float at4(const float4& v, int j) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); }

__device__ __forceinline__ float relax_f32(float xp, float xm, float yp, float ym, float zp, float zm, float b, float c,
                                           float omega, float dx2) {
    const float sum = xp + xm + yp + ym + zp + zm;
    const float pgs = (sum - b * dx2) * dev::kInv6;
    return c + omega * (pgs - c);
}

template <int P>
__device__ __forceinline__ float4 relax_row_f32(float4 XP, float4 XM, float4 YP, float4 YM, float4 K, float ZC, float4 B,
                                                float4 C, float omega, float dx2) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float zm = P ? at4(K, j) : (j > 0 ? at4(K, j - 1) : ZC);
        const float zp = P ? (j < 3 ? at4(K, j + 1) : ZC) : at4(K, j);
        v[j] = relax_f32(at4(XP, j), at4(XM, j), at4(YP, j), at4(YM, j), zp, zm, at4(B, j), at4(C, j), omega, dx2);
    }
    return make_float4(v[0], v[1], v[2], v[3]);
}

// relax_group on FP32 (see there): a pass over the kF32LeavesPerGroup leaves of group g; dx2
// scales the right-hand side.
constexpr int kF32LeavesPerGroup = kF32LeavesPerBlock * kF32LeavesPerThread;

template <bool kZero, bool kShared, bool kPdl, typename Mid>
__device__ __forceinline__ void relax_group_f32(const int* __restrict__ nb8, const float* __restrict__ rhs, float* e,
                                                int num_leaves, int g, int colour, float omega, float dx2, Mid&& mid) {
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) & 1;
    const int a = lane >> 2, b = 2 * (lane & 3) + ((a + w) & 1);
    const int p = (w + colour) & 1;
    const uint32_t rowc = ((uint32_t)colour << 8) | (uint32_t)(4 * (32 * w + lane));
    auto lde = [](const float* q) { return kShared ? ldf4_rw(q) : ldf4(q); };
    const int leaf0 = g * kF32LeavesPerGroup + (int)(threadIdx.x >> 6);
    uint32_t own[kF32LeavesPerThread];
    bool live[kF32LeavesPerThread];
#pragma unroll
    for (int k = 0; k < kF32LeavesPerThread; ++k) {
        const int leaf = leaf0 + k * kF32LeavesPerBlock;
        live[k] = leaf < num_leaves;
        own[k] = ((uint32_t)(live[k] ? leaf : 0) << 9) | rowc;
    }
    float4 B[kF32LeavesPerThread], out[kF32LeavesPerThread];
#pragma unroll
    for (int k = 0; k < kF32LeavesPerThread; ++k) B[k] = ldf4(rhs + own[k]);
    if constexpr (kZero) {
        mid();
#pragma unroll
        for (int k = 0; k < kF32LeavesPerThread; ++k) {
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = relax_f32(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, at4(B[k], j), 0.f, omega, dx2);
            out[k] = make_float4(v[0], v[1], v[2], v[3]);
            if (live[k]) *reinterpret_cast<float4*>(e + (own[k] ^ 256u)) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    } else {
        const uint32_t co = ((uint32_t)(colour ^ 1) << 8) | (uint32_t)(128 * (w ^ 1));
        auto row = [&](uint32_t n, int a2, int b2) { return (n << 9) | co | (uint32_t)(16 * a2 + 4 * (b2 >> 1)); };
        const int sx = a == 7 ? 0 : a == 0 ? 1 : 6, sy = b == 7 ? 2 : b == 0 ? 3 : 6, sz = 5 - p;
        uint32_t nx[kF32LeavesPerThread], ny[kF32LeavesPerThread], nz[kF32LeavesPerThread];
#pragma unroll
        for (int k = 0; k < kF32LeavesPerThread; ++k) {
            const int* nb = nb8 + 8 * (own[k] >> 9);
            nx[k] = (uint32_t)__ldg(nb + sx);
            ny[k] = (uint32_t)__ldg(nb + sy);
            nz[k] = (uint32_t)__ldg(nb + sz);
        }
        if constexpr (kPdl) asm volatile("griddepcontrol.wait;" ::: "memory");
        float4 C[kF32LeavesPerThread], K[kF32LeavesPerThread], XP[kF32LeavesPerThread], XM[kF32LeavesPerThread],
            YP[kF32LeavesPerThread], YM[kF32LeavesPerThread];
        float ZC[kF32LeavesPerThread];
#pragma unroll
        for (int k = 0; k < kF32LeavesPerThread; ++k) {
            C[k] = ldf4_rw(e + own[k]);
            K[k] = lde(e + (own[k] ^ 256u));
        }
#pragma unroll
        for (int k = 0; k < kF32LeavesPerThread; ++k) {
            const uint32_t lf = own[k] >> 9;
            XP[k] = lde(e + row(a == 7 ? nx[k] : lf, (a + 1) & 7, b));
            XM[k] = lde(e + row(a == 0 ? nx[k] : lf, (a - 1) & 7, b));
            YP[k] = lde(e + row(b == 7 ? ny[k] : lf, a, (b + 1) & 7));
            YM[k] = lde(e + row(b == 0 ? ny[k] : lf, a, (b - 1) & 7));
            const float* zq = e + ((nz[k] << 9) | ((own[k] ^ 256u) & 511u)) + 3u * (uint32_t)(p ^ 1);
            ZC[k] = kShared ? *zq : __ldg(zq);
        }
        mid();  // every load of the pass is in flight
#pragma unroll
        for (int k = 0; k < kF32LeavesPerThread; ++k)
            out[k] = p ? relax_row_f32<1>(XP[k], XM[k], YP[k], YM[k], K[k], ZC[k], B[k], C[k], omega, dx2)
                       : relax_row_f32<0>(XP[k], XM[k], YP[k], YM[k], K[k], ZC[k], B[k], C[k], omega, dx2);
    }
#pragma unroll
    for (int k = 0; k < kF32LeavesPerThread; ++k)
        if (live[k]) *reinterpret_cast<float4*>(e + own[k]) = out[k];
}

// rbgs_split_half_kernel on FP32 (see there).
template <bool kZero>
__global__ void __launch_bounds__(kF32Threads, kF32ShortGridCtasPerSm)
    rbgs_split_half_f32_kernel(const int* __restrict__ nb8, const float* __restrict__ rhs, float* e, int num_leaves,
                               int colour, float omega, float dx2, const double* __restrict__ check, double tol2,
                               unsigned long long* __restrict__ counters) {
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    if (counters != nullptr && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(counters, 1ull);
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int groups = (num_leaves + kF32LeavesPerGroup - 1) / kF32LeavesPerGroup;
    for (int g = blockIdx.x; g < groups; g += gridDim.x)
        relax_group_f32<kZero, false, true>(nb8, rhs, e, num_leaves, g, colour, omega, dx2, [] {});
}

// ---- The persistent solve -------------------------------------------------------------------
// A whole solve, `half_sweeps` half-sweeps (red, black, red, ...), in one cooperative launch
// instead of one launch per colour: no launch gap and no draining of a grid between the
// colours. Work item i = h * groups + g is half-sweep h of leaf group g; CTA c takes the items
// c, c + G, c + 2G, ... in order (G CTAs, all resident). Before item (h, g) the CTA waits until
// progress[x] >= h for g itself and for every group x that holds a face neighbour of g's leaves:
// those groups have finished half-sweep h - 1, so the other colour the item reads is current and
// no neighbour still has to read the colour the item overwrites. A done item is published as
// progress[g] = h + 1 (its stores fenced first) by its CTA during the CTA's next pass, once that
// pass's loads are in flight, so that the fence costs no time of its own; or at once, before the
// CTA waits for anything. The next item's dependencies are polled during the current pass too.
// The values are those of the launch-per-colour kernel to the bit: each voxel sees the same
// operands in the same order.
//
// Every wait ends: an item waits only on smaller items; a CTA publishes its done items before it
// waits, and one that does not wait publishes them during its next pass; so the smallest item
// not yet published belongs to a CTA that is working on it or about to publish it. Waits are
// bounded all the same (kSolveMaxPolls polls with a short sleep, about a second): one that gives
// up raises the device error flag (counters[1]) and the abort word progress[groups], which every
// other wait watches, and every CTA returns, leaving e unfinished. `unreachable` (0 but in the
// test of that path) raises every wait's target out of reach.
constexpr uint32_t kSolveMaxPolls = 1u << 20;
static_assert(kThreads == kF32Threads, "one block shape for both precisions");
static_assert(64 + 6 * kLeavesPerGroup + 1 <= kThreads, "dependency threads");

__device__ __forceinline__ uint32_t ld_acquire_u32(const unsigned* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(unsigned* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// T = __half: the FP16 inner solve (relax_group, unit spacing); T = float: the FP32 solve
// (relax_group_f32, dx2). Groups of kLeavesPerGroup or kF32LeavesPerGroup leaves.
template <typename T, bool kZeroFirst>
__global__ void __launch_bounds__(kThreads, kShortGridCtasPerSm) rbgs_split_solve_kernel(
    const int* __restrict__ nb8, const T* __restrict__ rhs, T* e, int num_leaves, int half_sweeps, float omega, float dx2,
    const double* __restrict__ check, double tol2, unsigned long long* __restrict__ counters, unsigned* progress,
    uint32_t max_polls, uint32_t unreachable) {
    constexpr bool kHalf = sizeof(T) == 2;
    constexpr int kPerGroup = kHalf ? kLeavesPerGroup : kF32LeavesPerGroup;
    constexpr int kDepThreads = 6 * kPerGroup;  // one face of one leaf each, threads 64 ...
    if (check != nullptr && check[0] <= tol2 * check[1]) return;  // the refinement has converged
    if (counters != nullptr && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(counters, (unsigned long long)half_sweeps);
    const int tid = threadIdx.x;
    const int groups = (num_leaves + kPerGroup - 1) / kPerGroup;
    unsigned* abort_word = progress + groups;
    const int64_t items = (int64_t)half_sweeps * groups;
    // The dependency this thread watches: face df of leaf dl of the item's group (threads 64 ...),
    // or the group itself (the thread after them); -1: none (and none in half-sweep 0).
    const int dt = tid - 64, dl = dt / 6, df = dt - 6 * dl;
    const bool watches_face = dt >= 0 && dt < kDepThreads, watches_self = dt == kDepThreads;
    auto dependency = [&](int h, int g) -> int {
        if (h == 0) return -1;
        if (watches_face) {
            const int leaf = g * kPerGroup + dl;
            if (leaf >= num_leaves) return -1;
            const int n = __ldg(nb8 + 8 * leaf + df);
            return n < num_leaves ? n / kPerGroup : -1;  // the zero leaf is never written
        }
        return watches_self ? g : -1;
    };
    auto publish = [&](int h, int g) {  // thread 0, after a CTA barrier that follows the item's stores
        __threadfence();
        st_relaxed_u32(progress + g, (uint32_t)(h + 1));
    };
    int h = (int)(blockIdx.x / (unsigned)groups), g = (int)(blockIdx.x % (unsigned)groups);
    const int step_h = (int)(gridDim.x / (unsigned)groups), step_g = (int)(gridDim.x % (unsigned)groups);
    int x = dependency(h, g);
    bool ok = x < 0 || ld_acquire_u32(progress + x) >= (uint32_t)h + unreachable;
    // The CTA's previous item, done but not yet published (ph < 0: none). Its publication waits
    // for a fence; it is deferred into the next item's pass, after that pass's loads are issued,
    // unless the next item has to wait (then it comes first: another CTA may wait for it).
    int ph = -1, pg = 0;
    for (int64_t i = blockIdx.x; i < items; i += gridDim.x) {
        // The previous item of this CTA is complete for this CTA's threads (its stores precede
        // the barrier below): a dependency on it needs no wait.
        if (!ok && x == pg && h - 1 == ph) ok = true;
        if (__syncthreads_or(!ok)) {
            if (tid == 0 && ph >= 0) publish(ph, pg);
            ph = -1;
            bool failed = false;
            if (!ok) {
                uint32_t polls = 0;
                while (ld_acquire_u32(progress + x) < (uint32_t)h + unreachable) {
                    if (++polls >= max_polls) {
                        atomicExch(abort_word, 1u);
                        if (counters != nullptr) atomicExch(counters + 1, 1ull);
                        failed = true;
                        break;
                    }
                    if ((polls & 31u) == 0 && *reinterpret_cast<volatile unsigned*>(abort_word) != 0u) {
                        failed = true;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            if (__syncthreads_or(failed)) return;
        }
        // The next item, and this thread's dependency of it, polled while this pass's loads are
        // in flight.
        int nh = h + step_h, ng = g + step_g;
        if (ng >= groups) ng -= groups, ++nh;
        const int nx = i + gridDim.x < items ? dependency(nh, ng) : -1;
        bool nok = true;
        auto mid = [&] {
            if (tid == 0 && ph >= 0) publish(ph, pg);
            if (nx >= 0) nok = ld_acquire_u32(progress + nx) >= (uint32_t)nh + unreachable;
        };
        if constexpr (kHalf) {
            if (kZeroFirst && h == 0)
                relax_group<true, true, false>(nb8, rhs, e, num_leaves, g, 0, omega, mid);
            else
                relax_group<false, true, false>(nb8, rhs, e, num_leaves, g, h & 1, omega, mid);
        } else {
            if (kZeroFirst && h == 0)
                relax_group_f32<true, true, false>(nb8, rhs, e, num_leaves, g, 0, omega, dx2, mid);
            else
                relax_group_f32<false, true, false>(nb8, rhs, e, num_leaves, g, h & 1, omega, dx2, mid);
        }
        ph = h, pg = g;
        h = nh, g = ng, x = nx, ok = nok;
    }
    __syncthreads();
    if (tid == 0 && ph >= 0) publish(ph, pg);
}

// Entry base of the half row (z = 4h .. 4h + 3) that starts at slot q (a multiple of 4), in the
// colour block of its z = 4h voxel, and that colour (p0); z = 4h + 1 and 4h + 3 sit at the same
// entries of the other colour.
__device__ __forceinline__ int64_t split_base(int64_t q, int& p0) {
    const int loc = (int)(q & 511), a = loc >> 6, b = (loc >> 3) & 7, h = (loc >> 2) & 1;
    p0 = (a + b) & 1;
    return (q & ~int64_t(511)) + 4 * (32 * p0 + 4 * a + (b >> 1)) + 2 * h;
}

// FP32 slot order <-> colour-split order, four values per thread.
__global__ void __launch_bounds__(256) to_split_f32_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < (n >> 2); u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = u << 2;
        int p0;
        const int64_t base = split_base(q, p0);
        const float4 v = __ldg(reinterpret_cast<const float4*>(src + q));
        *reinterpret_cast<float2*>(dst + base + ((int64_t)p0 << 8)) = make_float2(v.x, v.z);
        *reinterpret_cast<float2*>(dst + base + ((int64_t)(p0 ^ 1) << 8)) = make_float2(v.y, v.w);
    }
}

__global__ void __launch_bounds__(256) from_split_f32_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t n) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < (n >> 2); u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = u << 2;
        int p0;
        const int64_t base = split_base(q, p0);
        const float2 x = __ldg(reinterpret_cast<const float2*>(src + base + ((int64_t)p0 << 8)));
        const float2 y = __ldg(reinterpret_cast<const float2*>(src + base + ((int64_t)(p0 ^ 1) << 8)));
        *reinterpret_cast<float4*>(dst + q) = make_float4(x.x, y.x, x.y, y.y);
    }
}

// The FP64 residual {sum r^2, sum b^2} of the iterate e (FP32, colour-split), r = div dx^2 -
// (x+ + x- + y+ + y- + z+ + z- - 6 p), the staged kernel's residual per voxel, into acc. One
// thread per row of a leaf (both colours, 8 voxels), 2 leaves per CTA, one wave looping; returns
// at once when `check` has passed.
__global__ void __launch_bounds__(128) split_residual_f32_kernel(const int* __restrict__ nb8, const float* __restrict__ rhs,
                                                                 const float* __restrict__ e, int num_leaves, double h2,
                                                                 const double* __restrict__ check, double tol2,
                                                                 double* __restrict__ acc) {
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int r = threadIdx.x & 63, a = r >> 3, b = r & 7, par = (a + b) & 1;
    const uint32_t rp = (uint32_t)(4 * (32 * par + 4 * a + (b >> 1)));  // this row's entries in each colour block
    auto rowpos = [](int a2, int b2) { return (uint32_t)(4 * (32 * ((a2 + b2) & 1) + 4 * a2 + (b2 >> 1))); };
    // The row's 8 values from its two colour blocks: z = 2 j + ((a + b + c) & 1) is entry j of colour c.
    auto row8 = [&](uint32_t leaf, uint32_t pos, int parity, float v[8]) {
        const float4 c0 = ldf4(e + (leaf << 9) + pos), c1 = ldf4(e + (leaf << 9) + 256u + pos);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[2 * j + parity] = at4(c0, j);
            v[2 * j + (parity ^ 1)] = at4(c1, j);
        }
    };
    double r2 = 0.0, b2 = 0.0;
    const int groups = (num_leaves + 1) / 2;
    for (int g = blockIdx.x; g < groups; g += gridDim.x) {
        const int leaf = 2 * g + (int)(threadIdx.x >> 6);
        if (leaf >= num_leaves) continue;
        const int* nb = nb8 + 8 * leaf;
        const uint32_t lf = (uint32_t)leaf;
        const uint32_t nxp = a == 7 ? (uint32_t)__ldg(nb + 0) : lf, nxm = a == 0 ? (uint32_t)__ldg(nb + 1) : lf;
        const uint32_t nyp = b == 7 ? (uint32_t)__ldg(nb + 2) : lf, nym = b == 0 ? (uint32_t)__ldg(nb + 3) : lf;
        const uint32_t nzp = (uint32_t)__ldg(nb + 4), nzm = (uint32_t)__ldg(nb + 5);
        float c[8], xp[8], xm[8], yp[8], ym[8], bv[8];
        row8(lf, rp, par, c);
        row8(nxp, rowpos((a + 1) & 7, b), par ^ 1, xp);
        row8(nxm, rowpos((a - 1) & 7, b), par ^ 1, xm);
        row8(nyp, rowpos(a, (b + 1) & 7), par ^ 1, yp);
        row8(nym, rowpos(a, (b - 1) & 7), par ^ 1, ym);
        {
            const float4 c0 = ldf4(rhs + (lf << 9) + rp), c1 = ldf4(rhs + (lf << 9) + 256u + rp);
#pragma unroll
            for (int j = 0; j < 4; ++j) bv[2 * j + par] = at4(c0, j), bv[2 * j + (par ^ 1)] = at4(c1, j);
        }
        // Across the z faces: z = 7 of the -z leaf's row (entry 3 of colour (a + b + 1) & 1), z = 0
        // of the +z leaf's row (entry 0 of colour (a + b) & 1).
        const float zlo = __ldg(e + (nzm << 9) + ((uint32_t)(par ^ 1) << 8) + rp + 3u);
        const float zhi = __ldg(e + (nzp << 9) + ((uint32_t)par << 8) + rp);
#pragma unroll
        for (int z = 0; z < 8; ++z) {
            const double lap = (double)xp[z] + (double)xm[z] + (double)yp[z] + (double)ym[z] +
                               (double)(z < 7 ? c[z + 1] : zhi) + (double)(z > 0 ? c[z - 1] : zlo) - 6.0 * (double)c[z];
            const double bb = (double)bv[z] * h2;
            r2 += (bb - lap) * (bb - lap);
            b2 += bb * bb;
        }
    }
    __shared__ double red[2][4];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        b2 += __shfl_xor_sync(0xffffffffu, b2, o);
    }
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = r2, red[1][threadIdx.x >> 5] = b2;
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(acc, red[0][0] + red[0][1] + red[0][2] + red[0][3]);
        atomicAdd(acc + 1, red[1][0] + red[1][1] + red[1][2] + red[1][3]);
    }
}

}  // namespace

int* Context::split_faces() {
    int* nb8 = reinterpret_cast<int*>(scratch_f32("split_faces", (size_t)topo.num_leaves * 8));
    if (split_faces_built != nb8) {
        launch_split_face_table(*this, nb8);
        if (!stream_capturing()) split_faces_built = nb8;
    }
    return nb8;
}

void* Context::split_e(const char* name, size_t bytes, int which) {
    const size_t n = (size_t)num_voxels();
    char* e = reinterpret_cast<char*>(scratch_f32(name, ((n + 512) * bytes + 3) / 4));
    if (split_zero_leaf[which] != e) {
        HNS_CUDA(cudaMemsetAsync(e + n * bytes, 0, 512 * bytes, stream));
        if (!stream_capturing()) split_zero_leaf[which] = e;
    }
    return e;
}

void launch_split_face_table(const Context& c, int* nb8) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    split_face_table_kernel<<<(unsigned)((L + 255) / 256), 256, 0, c.stream>>>(c.topo.view, reinterpret_cast<int4*>(nb8));
    HNS_LAUNCHED();
}

void launch_rbgs_split_half(const Context& c, const int* nb8, const void* rhs, void* e, int colour, bool e_zero,
                            float omega, const double* check, double tol2, bool short_grid) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    if (L >= (int64_t(1) << 22)) fail(HNS_ERR_INVALID_ARG, "too many leaves for the colour-split inner solve");
    const int per_block = kLeavesPerBlock * kLeavesPerThread;
    unsigned blocks = (unsigned)((L + per_block - 1) / per_block);
    // A launch that will most likely return at once (the refinement expected to have converged)
    // uses one wave of CTAs: its cost is then the launch, not the scheduling of every CTA.
    if (short_grid) blocks = std::min(blocks, (unsigned)(c.sm_count() * kHalfCtasPerSm));
    const auto* r = static_cast<const __half*>(rhs);
    auto* x = static_cast<__half*>(e);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[2];
    unsigned na = 0;
    if (e_zero) {
        cfg.numAttrs = c.add_inner_window(attr, 0);
        cfg.attrs = attr;
        HNS_CUDA(cudaLaunchKernelEx(&cfg, rbgs_split_half_kernel<true>, nb8, r, x, (int)L, colour, omega, check, tol2,
                                    c.counters));
        HNS_LAUNCHED();
        return;
    }
    // Programmatic dependent launch: the sweep's prologue (the convergence check, the face table
    // and the right-hand side) overlaps the tail of the preceding half-sweep, and e is read after
    // griddepcontrol.wait. The caller guarantees that the preceding kernel on the stream is a
    // half-sweep and that rhs, nb8 and check were written before it started.
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
    na = c.add_inner_window(attr, na);
    cfg.attrs = attr;
    cfg.numAttrs = na;
    HNS_CUDA(cudaLaunchKernelEx(&cfg, rbgs_split_half_kernel<false>, nb8, r, x, (int)L, colour, omega, check, tol2,
                                c.counters));
    HNS_LAUNCHED();
}

namespace {

template <typename T>
void launch_split_solve(Context& c, const int* nb8, const T* rhs, T* e, int half_sweeps, bool e_zero, float omega,
                        float dx2, const double* check, double tol2) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0 || half_sweeps <= 0) return;
    if (L >= (int64_t(1) << 22)) fail(HNS_ERR_INVALID_ARG, "too many leaves for the colour-split solve");
    const int per_group = sizeof(T) == 2 ? kLeavesPerGroup : kF32LeavesPerGroup;
    const int groups = (int)((L + per_group - 1) / per_group);
    // Progress counters of the leaf groups and the abort word, zero before each launch.
    auto* progress = reinterpret_cast<unsigned*>(
        c.scratch_f32(sizeof(T) == 2 ? "split_progress16" : "split_progress32", (size_t)groups + 1));
    HNS_CUDA(cudaMemsetAsync(progress, 0, sizeof(unsigned) * ((size_t)groups + 1), c.stream));
    auto kern = e_zero ? rbgs_split_solve_kernel<T, true> : rbgs_split_solve_kernel<T, false>;
    int per_sm = 0;
    HNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0));
    if (per_sm < 1) fail(HNS_ERR_CUDA, "the persistent solve does not fit on an SM");
    // At most one CTA per group: a CTA beyond that could only hold an item of a later half-sweep
    // and wait for it.
    const unsigned blocks = (unsigned)std::min<int64_t>(groups, (int64_t)per_sm * c.sm_count());
    // The test hook: every wait gives up after first_wait_polls polls, its target out of reach.
    const bool stall = c.first_wait_polls >= 0;
    const uint32_t max_polls = stall ? (uint32_t)c.first_wait_polls : kSolveMaxPolls;
    const uint32_t unreachable = stall ? (1u << 30) : 0u;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads);
    cfg.stream = c.stream;
    // Cooperative: every CTA resident at once, which the progress waits rely on.
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HNS_CUDA(cudaLaunchKernelEx(&cfg, kern, nb8, rhs, e, (int)L, half_sweeps, omega, dx2, check, tol2, c.counters,
                                progress, max_polls, unreachable));
    HNS_LAUNCHED();
}

}  // namespace

void launch_rbgs_split_solve(Context& c, const int* nb8, const void* rhs, void* e, int half_sweeps, bool e_zero,
                             float omega, const double* check, double tol2) {
    launch_split_solve(c, nb8, static_cast<const __half*>(rhs), static_cast<__half*>(e), half_sweeps, e_zero, omega, 1.0f,
                       check, tol2);
}

void launch_rbgs_split_solve_f32(Context& c, const int* nb8, const float* rhs, float* e, int half_sweeps, bool e_zero,
                                 float omega, float dx2, const double* check, double tol2) {
    launch_split_solve(c, nb8, rhs, e, half_sweeps, e_zero, omega, dx2, check, tol2);
}

}  // namespace hns

namespace hns {

void launch_rbgs_split_half_f32(const Context& c, const int* nb8, const float* rhs, float* e, int colour, bool e_zero,
                                float omega, float dx2, const double* check, double tol2, bool short_grid, bool pdl) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    if (L >= (int64_t(1) << 22)) fail(HNS_ERR_INVALID_ARG, "too many leaves for the colour-split solve");
    const int per_block = kF32LeavesPerBlock * kF32LeavesPerThread;
    unsigned blocks = (unsigned)((L + per_block - 1) / per_block);
    if (short_grid) blocks = std::min(blocks, (unsigned)(c.sm_count() * kF32ShortGridCtasPerSm));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kF32Threads);
    cfg.stream = c.stream;
    if (e_zero) {
        HNS_CUDA(cudaLaunchKernelEx(&cfg, rbgs_split_half_f32_kernel<true>, nb8, rhs, e, (int)L, colour, omega, dx2, check,
                                    tol2, c.counters));
        HNS_LAUNCHED();
        return;
    }
    if (!pdl) {
        HNS_CUDA(cudaLaunchKernelEx(&cfg, rbgs_split_half_f32_kernel<false>, nb8, rhs, e, (int)L, colour, omega, dx2, check,
                                    tol2, c.counters));
        HNS_LAUNCHED();
        return;
    }
    // Programmatic dependent launch, as the FP16 half-sweep (launch_rbgs_split_half).
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HNS_CUDA(cudaLaunchKernelEx(&cfg, rbgs_split_half_f32_kernel<false>, nb8, rhs, e, (int)L, colour, omega, dx2, check,
                                tol2, c.counters));
    HNS_LAUNCHED();
}

void convert_split_f32(const Context& c, const float* src, float* dst, bool to_split) {
    const int64_t n = c.num_voxels();
    if (n == 0) return;
    const unsigned g = (unsigned)std::min<int64_t>((n / 4 + 255) / 256, (int64_t)c.sm_count() * 16);
    if (to_split)
        to_split_f32_kernel<<<g, 256, 0, c.stream>>>(src, dst, n);
    else
        from_split_f32_kernel<<<g, 256, 0, c.stream>>>(src, dst, n);
    HNS_LAUNCHED();
}

void launch_split_residual_f32(const Context& c, const int* nb8, const float* rhs, const float* e, double h2,
                               const double* check, double tol2, double* acc) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    const unsigned g = (unsigned)std::min<int64_t>((L + 1) / 2, (int64_t)c.sm_count() * 8);
    split_residual_f32_kernel<<<g, 128, 0, c.stream>>>(nb8, rhs, e, (int)L, h2, check, tol2, acc);
    HNS_LAUNCHED();
}

}  // namespace hns
