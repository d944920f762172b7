// The red-black SOR iteration on colour-packed FP16 rows, staged by TMA: the inner solve of
// the mixed-precision refinement (L e = r with unit spacing, e and r in FP16, FP32 arithmetic).
//
// Layout. The inner solve's arrays belong to the solver, so their layout is free. Each z-row of
// a leaf is stored colour-packed: the values at z = 0, 2, 4, 6 and then at z = 1, 3, 5, 7
// (position of z = (z & 1) * 4 + (z >> 1)). The red voxels of a row are then one contiguous
// half-row and the black voxels the other, and a lane updates two voxels of one colour from
// one 4-byte load per neighbour row: a warp's load moves 64 useful values per shared-memory
// wavefront where a scalar FP16 load moves 32.
//
// Staging. The arrays are viewed as 4-D tensors [leaf][x][y][z] of FP16 with 16-byte rows, and
// one thread stages a leaf's stencil with 26 TMA box loads (cp.async.bulk.tensor, no multicast):
// the leaf, x-face pairs, y-face pairs, the xy-edge rows, the two z-neighbour leaves with the
// ring rows their x/y neighbours hold, and the right-hand side with its one-voxel halo. A
// missing neighbour is the leaf coordinate -1, which TMA fills with zeros (the reference's
// p = 0 outside the domain). Every box lands densely at a 128-byte-aligned offset.
//
// Per leaf, the update is one full iteration of redBlackGaussSeidelUpdate
// (src/Cuda/Kernel.cu:459-489) -- red on the leaf and its one-voxel face ring, then black on
// the leaf -- with the arithmetic, operation order and FP16 rounding points of
// rbgs_stream_kernel<__half> in hns_rbgs.cu, so both produce the same values to the bit (the
// tests compare them). The kernel is persistent: CTA g relaxes leaves g, g + G, ..., with
// kStages shared-memory stages so that the boxes of the next leaves are in flight while one
// is relaxed.
//
// Work of a lane: warp w owns leaf rows (a, b) with a in {2w, 2w+1}, lane = 16 (a - 2w) +
// 2 b + m, and updates the pair m (voxels 2m, 2m+1 of the colour's half-row):
//   * red: the pair from the four x/y neighbour rows and the row's own black half (one 8-byte
//     load gives all its z-neighbours), and the row's red z-ring voxel (z = 8 if a + b is even,
//     else z = -1), which only this row's black voxels need, so it stays in a register;
//   * black: the pair from the neighbour rows' updated red halves, the lane's own red pair and
//     its partner lane's (a shuffle), and the z-ring voxel; both pairs go straight to HBM.
// Warps 2 and 3 also relax the red voxels of the x-ring rows (a = -1, 8) and the y-ring rows
// (b = -1, 8), when the leaf on that side exists.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "hns_internal.cuh"
#include "hns_ptx.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace pk {

constexpr int NC = 128;      // consumer threads (4 warps): the relaxation
constexpr int NT = NC + 32;  // + one producer warp: the neighbour tables and the TMA boxes
constexpr int kMinBlocksPerSM = 7;
// Shared-memory stages: a CTA's boxes run kStages - 1 leaves ahead of its relaxation.
constexpr int kStages = 3;
// Bounded mbarrier wait: give up after kWaitCycles SM cycles (about 1 s at 2 GHz).
constexpr long long kWaitCycles = 2000000000LL;

__host__ __device__ constexpr int nbi(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }
__host__ __device__ constexpr int parity(int a, int b) { return (a + b) & 1; }  // two's complement: ok for -1

// ---- stage layout (bytes; a row is 16 bytes = 8 packed FP16 values) -------------------------
//   E    e rows (a, b), a in [-2, 9] (12 planes of 8 rows), b in [0, 8)
//   YM   e rows (a, b), a in [0, 8), b in {-2, -1}: [a][2]
//   YP   e rows (a, b), a in [0, 8), b in {8, 9}: [a][2]
//   YE   e rows of the four xy-edge columns, one 128-byte slot each: (-1, {-2,-1}),
//        (8, {-2,-1}), (-1, {8,9}), (8, {8,9})
//   ZM   rows of the -z leaf: (a, b) for a in [-1, 8], b in [0, 8) (10 planes), then the rows
//        (a, -1) and (a, 8), a in [0, 8) -- z = -1 is at row position 7, z = -2 at 3
//   ZP   the same for the +z leaf -- z = 8 at position 0, z = 9 at 4
//   B    right-hand-side rows (a, b), a in [-1, 8], b in [0, 8); then (a, -1), (a, 8)
//   BZM  the -z leaf's right-hand side (a, b), a, b in [0, 8); BZP the +z leaf's
constexpr int kOffE = 0;
constexpr int kOffYM = kOffE + 12 * 128;
constexpr int kOffYP = kOffYM + 256;
constexpr int kOffYE = kOffYP + 256;
constexpr int kOffZM = kOffYE + 4 * 128;
constexpr int kZPlanes = 10 * 128;       // planes a = -1..8
constexpr int kZBytes = kZPlanes + 256;  // + rows (a, -1) and (a, 8)
constexpr int kOffZP = kOffZM + kZBytes;
constexpr int kOffB = kOffZP + kZBytes;
constexpr int kOffBYM = kOffB + 10 * 128;
constexpr int kOffBYP = kOffBYM + 128;
constexpr int kOffBZM = kOffBYP + 128;
constexpr int kOffBZP = kOffBZM + 1024;
constexpr int kStageBytes = kOffBZP + 1024;

// Byte offset of e row (a, b) in a stage: a in [-2, 9] for b in [0, 8); otherwise the y-face
// and edge rows listed above.
__host__ __device__ constexpr int e_row(int a, int b) {
    return (b >= 0 && b < 8) ? kOffE + (a + 2) * 128 + b * 16
           : (a >= 0 && a < 8) ? (b < 0 ? kOffYM + a * 32 + (b + 2) * 16 : kOffYP + a * 32 + (b - 8) * 16)
           : kOffYE + ((a < 0 ? 0 : 1) + (b < 0 ? 0 : 2)) * 128 + (b < 0 ? b + 2 : b - 8) * 16;
}
// Row (a, b) of the -z (zoff = kOffZM) or +z (kOffZP) leaf: a in [-1, 8] for b in [0, 8);
// b = -1 or 8 for a in [0, 8).
__host__ __device__ constexpr int z_row(int zoff, int a, int b) {
    return (b >= 0 && b < 8) ? zoff + (a + 1) * 128 + b * 16 : zoff + kZPlanes + (b < 0 ? 0 : 128) + a * 16;
}
// Right-hand-side row (a, b) of the leaf: a in [-1, 8] for b in [0, 8); b = -1 or 8 for a in [0, 8).
__host__ __device__ constexpr int b_row(int a, int b) {
    return (b >= 0 && b < 8) ? kOffB + (a + 1) * 128 + b * 16 : (b < 0 ? kOffBYM : kOffBYP) + a * 16;
}

struct __align__(128) Stage {
    uint4 data[kStageBytes / 16];
    uint64_t bar;  // completes when the stage's 26 boxes have landed
    int nb[27];    // the staged leaf's neighbour table
};

// ---- the boxes of one leaf -------------------------------------------------------------------
// Tensor maps (passed as one kernel parameter): e maps first, then right-hand-side maps. Box
// extents are (z, y, x, leaf); coordinates (0, y0, x0, neighbour leaf).
enum MapId : int {
    kMapFull = 0,   // e (8, 8, 8, 1)
    kMapXPair,      // e (8, 8, 2, 1)
    kMapXPlane,     // e (8, 8, 1, 1)
    kMapYPair,      // e (8, 2, 8, 1)
    kMapYRow,       // e (8, 1, 8, 1)
    kMapEdge,       // e (8, 2, 1, 1)
    kMapRFull,      // rhs (8, 8, 8, 1)
    kMapRXPlane,    // rhs (8, 8, 1, 1)
    kMapRYRow,      // rhs (8, 1, 8, 1)
    kNumMaps
};
constexpr int kBoxX[kNumMaps] = {8, 2, 1, 8, 8, 1, 8, 1, 8};
constexpr int kBoxY[kNumMaps] = {8, 8, 8, 2, 1, 2, 8, 8, 1};

struct TensorMaps {
    CUtensorMap m[kNumMaps];
};

struct Box {
    int map, y0, x0, q, dst;
};
constexpr int kBoxes = 26;

__host__ __device__ constexpr Box box(int i) {
    // clang-format off
    constexpr Box list[kBoxes] = {
        {kMapXPair, 0, 6, nbi(-1, 0, 0), e_row(-2, 0)},   // x-face planes a = -2, -1
        {kMapFull, 0, 0, nbi(0, 0, 0), e_row(0, 0)},      // the leaf
        {kMapXPair, 0, 0, nbi(1, 0, 0), e_row(8, 0)},     // x-face planes a = 8, 9
        {kMapYPair, 6, 0, nbi(0, -1, 0), e_row(0, -2)},   // y-face rows b = -2, -1
        {kMapYPair, 0, 0, nbi(0, 1, 0), e_row(0, 8)},     // y-face rows b = 8, 9
        {kMapEdge, 6, 7, nbi(-1, -1, 0), e_row(-1, -2)},  // xy-edge columns
        {kMapEdge, 6, 0, nbi(1, -1, 0), e_row(8, -2)},
        {kMapEdge, 0, 7, nbi(-1, 1, 0), e_row(-1, 8)},
        {kMapEdge, 0, 0, nbi(1, 1, 0), e_row(8, 8)},
        {kMapXPlane, 0, 7, nbi(-1, 0, -1), z_row(kOffZM, -1, 0)},  // -z leaf and its ring rows
        {kMapFull, 0, 0, nbi(0, 0, -1), z_row(kOffZM, 0, 0)},
        {kMapXPlane, 0, 0, nbi(1, 0, -1), z_row(kOffZM, 8, 0)},
        {kMapYRow, 7, 0, nbi(0, -1, -1), z_row(kOffZM, 0, -1)},
        {kMapYRow, 0, 0, nbi(0, 1, -1), z_row(kOffZM, 0, 8)},
        {kMapXPlane, 0, 7, nbi(-1, 0, 1), z_row(kOffZP, -1, 0)},   // +z leaf and its ring rows
        {kMapFull, 0, 0, nbi(0, 0, 1), z_row(kOffZP, 0, 0)},
        {kMapXPlane, 0, 0, nbi(1, 0, 1), z_row(kOffZP, 8, 0)},
        {kMapYRow, 7, 0, nbi(0, -1, 1), z_row(kOffZP, 0, -1)},
        {kMapYRow, 0, 0, nbi(0, 1, 1), z_row(kOffZP, 0, 8)},
        {kMapRXPlane, 0, 7, nbi(-1, 0, 0), b_row(-1, 0)},  // right-hand side, one-voxel halo
        {kMapRFull, 0, 0, nbi(0, 0, 0), b_row(0, 0)},
        {kMapRXPlane, 0, 0, nbi(1, 0, 0), b_row(8, 0)},
        {kMapRYRow, 7, 0, nbi(0, -1, 0), b_row(0, -1)},
        {kMapRYRow, 0, 0, nbi(0, 1, 0), b_row(0, 8)},
        {kMapRFull, 0, 0, nbi(0, 0, -1), kOffBZM},          // z-neighbour right-hand sides
        {kMapRFull, 0, 0, nbi(0, 0, 1), kOffBZP},
    };
    // clang-format on
    return list[i];
}

constexpr int box_bytes(int i) { return 8 * 2 * kBoxY[box(i).map] * kBoxX[box(i).map]; }
constexpr int stage_tx_bytes() {
    int s = 0;
    for (int i = 0; i < kBoxes; ++i) s += box_bytes(i);
    return s;
}
constexpr uint32_t kStageTx = stage_tx_bytes();

// Fixed shared-memory byte offsets (relative to a stage) of one thread's loads and stores.
struct LaneGeom {
    int a, b, m, pi;  // leaf row (a, b), pair m, parity of a + b
    int red;          // the row's red pair (E); x neighbours at +- 128
    int yp, ym;       // the y-neighbour rows' pairs at the red positions
    int dk;           // black positions - red positions (8 - 16 pi)
    int b_red;        // right-hand side of the red pair; the black pair's at + dk
    int zm7;          // z = -1 of the row (ZM row, position 7); z = 8 (ZP position 0) at + kZP0
    int zc;           // the row's red z-ring voxel (zp0 if pi = 0, else zm7); x neighbours at +- 128
    int zyp, zym;     // its y neighbours
    int zfar;         // its z-neighbour beyond: z = 9 if pi = 0, else z = -2
    int bz;           // right-hand side of the z-ring voxel
    int zq;           // neighbour-table index of the leaf holding the z-ring voxel
    int gout;         // byte offset of the row in a leaf's block
    // ring row (warps 2, 3): x-ring (a = -1, 8) for warp 2, y-ring (b = -1, 8) for warp 3
    int ra, rb, rpi;
    int rred, rxp, rxm, ryp, rym;  // its red pair and the neighbours' pairs at the same positions
    int rblack;                    // its black half (8 bytes)
    int rb_red;                    // right-hand side of the red pair
    int rhalo;                     // the z-halo its red voxels need: z = -1 if rpi = 0, else z = 8
    int rq;                        // neighbour-table index of the ring row's leaf
};
constexpr int kZP0 = kOffZP - kOffZM - 14;  // z_row(kOffZP, a, b) - (z_row(kOffZM, a, b) + 14)

__host__ __device__ inline LaneGeom lane_geom(int tid) {
    LaneGeom g{};
    const int lane = tid & 31, warp = tid >> 5;
    g.m = lane & 1;
    g.b = (lane >> 1) & 7;
    g.a = 2 * warp + (lane >> 4);
    g.pi = parity(g.a, g.b);
    const int pos = 8 * g.pi + 4 * g.m;
    g.red = e_row(g.a, g.b) + pos;
    g.yp = e_row(g.a, g.b + 1) + pos;
    g.ym = e_row(g.a, g.b - 1) + pos;
    g.dk = 8 - 16 * g.pi;
    g.b_red = b_row(g.a, g.b) + pos;
    g.zm7 = z_row(kOffZM, g.a, g.b) + 14;
    const int zoff = g.pi ? kOffZM : kOffZP, zpos = g.pi ? 14 : 0;
    g.zc = z_row(zoff, g.a, g.b) + zpos;
    g.zyp = z_row(zoff, g.a, g.b + 1) + zpos;
    g.zym = z_row(zoff, g.a, g.b - 1) + zpos;
    g.zfar = g.pi ? g.zc - 8 : g.zc + 8;
    g.bz = (g.pi ? kOffBZM + 14 : kOffBZP) + g.a * 128 + g.b * 16;
    g.zq = nbi(0, 0, g.pi ? -1 : 1);
    g.gout = (g.a * 64 + g.b * 8) * 2;
    const int side = lane >> 4, k = (lane >> 1) & 7;
    if (warp == 2) {
        g.ra = side ? 8 : -1, g.rb = k, g.rq = nbi(side ? 1 : -1, 0, 0);
    } else if (warp == 3) {
        g.ra = k, g.rb = side ? 8 : -1, g.rq = nbi(0, side ? 1 : -1, 0);
    } else {
        g.ra = 0, g.rb = 0, g.rq = nbi(0, 0, 0);  // unused
    }
    g.rpi = parity(g.ra, g.rb);
    const int rpos = 8 * g.rpi + 4 * g.m;
    g.rred = e_row(g.ra, g.rb) + rpos;
    g.rxp = e_row(g.ra + 1, g.rb) + rpos;
    g.rxm = e_row(g.ra - 1, g.rb) + rpos;
    g.ryp = e_row(g.ra, g.rb + 1) + rpos;
    g.rym = e_row(g.ra, g.rb - 1) + rpos;
    g.rblack = e_row(g.ra, g.rb) + 8 * (1 - g.rpi);
    g.rb_red = b_row(g.ra, g.rb) + rpos;
    g.rhalo = g.rpi ? z_row(kOffZP, g.ra, g.rb) : z_row(kOffZM, g.ra, g.rb) + 14;
    return g;
}

__device__ __forceinline__ uint32_t lds32(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t lds16(uint32_t a) {
    unsigned short v;
    asm volatile("ld.shared.b16 %0, [%1];" : "=h"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void lds64(uint32_t a, uint32_t& lo, uint32_t& hi) {
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "r"(a));
}
__device__ __forceinline__ void sts32(uint32_t a, uint32_t v) { asm volatile("st.shared.b32 [%0], %1;" ::"r"(a), "r"(v)); }

// FP16 operand (low 16 bits of h) into FP32 arithmetic: h + c, and a * b + c, rounded once.
__device__ __forceinline__ float addh(uint32_t h, float c) {
    float d;
    asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"((unsigned short)h), "f"(c));
    return d;
}
__device__ __forceinline__ float fmah(uint32_t a, uint32_t b, float c) {
    float d;
    asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"((unsigned short)a), "h"((unsigned short)b), "f"(c));
    return d;
}
__device__ __forceinline__ float h2f(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)h)); }

constexpr uint32_t kHalfMinusOne = 0xBC00u;

// One update of redBlackGaussSeidelUpdate with dx^2 = 1, as rbgs_stream_kernel<__half> does it:
// sum = x+ + x- + y+ + y- + z+ + z- (FP32, in that order), pgs = (sum - b) times the
// reference's 1/6, result = c + omega (pgs - c), rounded to FP16 by the caller. The FP16
// operands enter the FP32 operations directly (their conversion is exact).
__device__ __forceinline__ float relax1(uint32_t xp, uint32_t xm, uint32_t yp, uint32_t ym, uint32_t zp, uint32_t zm,
                                        uint32_t b, uint32_t c, float omega) {
    float s = h2f(xp);
    s = addh(xm, s);
    s = addh(yp, s);
    s = addh(ym, s);
    s = addh(zp, s);
    s = addh(zm, s);
    const float pgs = fmah(b, kHalfMinusOne, s) * dev::kInv6;  // (sum - b * 1) / 6
    const float d = fmah(c, kHalfMinusOne, pgs);              // pgs - c
    return addh(c, omega * d);                                 // c + omega (pgs - c)
}

// The same on the two halves of packed pairs; returns the packed FP16 results.
__device__ __forceinline__ uint32_t relax2(uint32_t xp, uint32_t xm, uint32_t yp, uint32_t ym, uint32_t zp, uint32_t zm,
                                           uint32_t b, uint32_t c, float omega) {
    const float lo = relax1(xp, xm, yp, ym, zp, zm, b, c, omega);
    const float hi = relax1(xp >> 16, xm >> 16, yp >> 16, ym >> 16, zp >> 16, zm >> 16, b >> 16, c >> 16, omega);
    const __half2 r = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&r);
}

__device__ __forceinline__ uint32_t round_half(float v) { return __half_as_ushort(__float2half_rn(v)); }

// The z-neighbour pairs of the lane's red pair from the row's black half (k01, k23) and the
// row's z = -1 / z = 8 values: with pi = 0 the red voxels are at even z and their z+ are the
// black values at the same index, their z- one index lower; with pi = 1 the other way round.
__device__ __forceinline__ void red_z_pairs(uint32_t k01, uint32_t k23, uint32_t zlo, uint32_t zhi, int m, int pi,
                                            uint32_t& zp, uint32_t& zm) {
    const uint32_t same = m ? k23 : k01;                     // black values 2m, 2m+1
    const uint32_t mid = __byte_perm(k01, k23, 0x5432);      // black values 1, 2
    const uint32_t lo_edge = __byte_perm(zlo, k01, 0x5410);  // z = -1, black value 0
    const uint32_t hi_edge = __byte_perm(k23, zhi, 0x5432);  // black value 3, z = 8
    const uint32_t shifted = (pi != m) ? mid : (pi ? hi_edge : lo_edge);
    zp = pi ? shifted : same;
    zm = pi ? same : shifted;
}

// Issues the 26 boxes of leaf `leaf` into stage S (one thread). e_zero: e = 0 (the first
// iteration of a solve), so every e box is read at leaf -1 and arrives as zeros.
__device__ __forceinline__ void stage_issue(Stage& S, const TensorMaps& maps, int e_zero) {
    const uint32_t base = ptx::smem_addr(&S);
    ptx::mbar_arrive_expect_tx(&S.bar, kStageTx);
#pragma unroll
    for (int i = 0; i < kBoxes; ++i) {
        const Box bx = box(i);
        const int leaf = (e_zero && bx.map < kMapRFull) ? -1 : S.nb[bx.q];
        ptx::tma_load_4d(base + bx.dst, &maps.m[bx.map], 0, bx.y0, bx.x0, leaf, &S.bar);
    }
}

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"r"(NC) : "memory"); }

// Consumers (warps 0-3): relax the CTA's leaves in order from the staged boxes.
__device__ __forceinline__ void consume(Stage* st, uint64_t* empty, int* cok, const LaneGeom& g, int tid, int64_t L,
                                        int64_t G, char* out, float omega, unsigned long long* counters) {
    const int warp = tid >> 5, lane = tid & 31;
    int64_t leaf = blockIdx.x;
    for (uint32_t j = 0; leaf < L; ++j, leaf += G) {
        const int s = j % kStages;
        Stage& cur = st[s];
        // One thread waits for the stage's boxes; the others wait at the consumer barrier, and
        // all of them read the outcome after it.
        if (tid == 0) {
            const bool landed = ptx::mbar_wait_bounded_clock(&cur.bar, (j / kStages) & 1, kWaitCycles);
            if (!landed && counters != nullptr) atomicExch(counters + 1, 1ull);
            *cok = landed ? 1 : 0;
        }
        consumer_sync();
        if (!*cok) return;  // e_out keeps its old values for the leaves left
        const uint32_t S = ptx::smem_addr(&cur);

        // ---- red ----
        uint32_t k01, k23;
        lds64(S + g.red - 4 * g.m + g.dk, k01, k23);  // the row's black half
        const uint32_t zm7 = lds16(S + g.zm7), zp0 = lds16(S + g.zm7 + kZP0);
        uint32_t zp, zm;
        red_z_pairs(k01, k23, zm7, zp0, g.m, g.pi, zp, zm);
        const uint32_t red = relax2(lds32(S + g.red + 128), lds32(S + g.red - 128), lds32(S + g.yp), lds32(S + g.ym), zp, zm,
                                    lds32(S + g.b_red), lds32(S + g.red), omega);
        sts32(S + g.red, red);
        // The row's red z-ring voxel: its x/y neighbours are the neighbour rows' values at the
        // same z; its z-neighbours are the row's black value at z = 7 (pi = 0) or z = 0 (pi = 1)
        // and the value beyond it.
        uint32_t zring;
        {
            const uint32_t near = g.pi ? (k01 & 0xffffu) : (k23 >> 16);
            const uint32_t far = lds16(S + g.zfar);
            const uint32_t ctr = g.pi ? zm7 : zp0;
            const float v = relax1(lds16(S + g.zc + 128), lds16(S + g.zc - 128), lds16(S + g.zyp), lds16(S + g.zym),
                                   g.pi ? near : far, g.pi ? far : near, lds16(S + g.bz), ctr, omega);
            zring = cur.nb[g.zq] >= 0 ? round_half(v) : ctr;
        }
        if (warp >= 2 && cur.nb[g.rq] >= 0) {  // ring rows
            uint32_t r01, r23;
            lds64(S + g.rblack, r01, r23);
            const uint32_t h = lds16(S + g.rhalo);
            uint32_t rzp, rzm;
            red_z_pairs(r01, r23, h, h, g.m, g.rpi, rzp, rzm);
            sts32(S + g.rred, relax2(lds32(S + g.rxp), lds32(S + g.rxm), lds32(S + g.ryp), lds32(S + g.rym), rzp, rzm,
                                     lds32(S + g.rb_red), lds32(S + g.rred), omega));
        }
        consumer_sync();

        // ---- black ----
        // z-neighbours: pi = 0 (black at odd z): z- = the red value at the same index, z+ = the
        // next one (the partner lane's first, or the z-ring voxel at z = 8); pi = 1 (black at
        // even z): z+ = the red value at the same index, z- = the previous one (the partner's
        // last, or the z-ring voxel at z = -1).
        const uint32_t other = __shfl_xor_sync(0xffffffffu, red, 1);
        uint32_t bzp, bzm;
        if (g.pi == 0) {
            bzm = red;
            bzp = __byte_perm(red, g.m ? zring : other, 0x5432);
        } else {
            bzp = red;
            bzm = __byte_perm(g.m ? other : (zring << 16), red, 0x5432);
        }
        const uint32_t cb = g.m ? k23 : k01;  // the lane's black pair, unchanged by the red sweep
        const uint32_t blk = relax2(lds32(S + g.red + g.dk + 128), lds32(S + g.red + g.dk - 128), lds32(S + g.yp + g.dk),
                                    lds32(S + g.ym + g.dk), bzp, bzm, lds32(S + g.b_red + g.dk), cb, omega);
        char* row = out + (leaf << 10) + g.gout;
        *reinterpret_cast<uint32_t*>(row + 8 * g.pi + 4 * g.m) = red;
        *reinterpret_cast<uint32_t*>(row + 8 * (1 - g.pi) + 4 * g.m) = blk;
        // This warp is done with the stage: order its reads and writes of it before the next
        // boxes (async proxy) and release it to the producer.
        ptx::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(&empty[s]);
    }
}

// Producer (warp 4): for each of the CTA's leaves, waits until the consumers have released the
// stage's previous leaf, writes the leaf's neighbour table into it and issues its 26 boxes.
// If a release never comes (the consumers stopped), it waits for its boxes still in flight so
// that none lands after the CTA has exited.
__device__ __forceinline__ void produce(Stage* st, uint64_t* empty, const TensorMaps& maps, const TopoView& t,
                                        int lane, int64_t L, int64_t G, int e_zero, unsigned long long* counters) {
    int64_t leaf = blockIdx.x;
    int nb_next = (lane < 27 && leaf < L) ? __ldg(t.nbr27 + leaf * 27 + lane) : -1;
    for (uint32_t j = 0; leaf < L; ++j, leaf += G) {
        const int s = j % kStages;
        const int nb = nb_next;
        nb_next = (lane < 27 && leaf + G < L) ? __ldg(t.nbr27 + (leaf + G) * 27 + lane) : -1;
        bool released = true;
        if (j >= kStages && lane == 0) released = ptx::mbar_wait_bounded_clock(&empty[s], (j / kStages - 1) & 1, kWaitCycles);
        released = __shfl_sync(0xffffffffu, released ? 1 : 0, 0) != 0;
        if (!released) {
            if (lane == 0) {
                if (counters != nullptr) atomicExch(counters + 1, 1ull);
                for (uint32_t k = j > kStages ? j - kStages : 0; k < j; ++k)
                    (void)ptx::mbar_wait_bounded_clock(&st[k % kStages].bar, (k / kStages) & 1, kWaitCycles);
            }
            return;
        }
        if (lane < 27) st[s].nb[lane] = nb;
        __syncwarp();
        if (lane == 0) stage_issue(st[s], maps, e_zero);
        __syncwarp();
    }
}

__global__ void __launch_bounds__(NT, kMinBlocksPerSM)
    rbgs_packed_kernel(const __grid_constant__ TensorMaps maps, TopoView t, __half* __restrict__ e_out, int e_zero,
                       float omega, const double* __restrict__ check, double tol2,
                       unsigned long long* __restrict__ counters) {
    __shared__ Stage st[kStages];
    __shared__ uint64_t empty[kStages];
    __shared__ int cok;
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int tid = threadIdx.x;
    const int64_t L = t.num_leaves, G = gridDim.x;
    if (tid == 0) {
        for (int k = 0; k < kStages; ++k) {
            ptx::mbar_init(&st[k].bar, 1);
            ptx::mbar_init(&empty[k], NC / 32);
        }
        ptx::fence_barrier_init();
        if (counters != nullptr && blockIdx.x == 0) atomicAdd(counters, 1ull);
    }
    __syncthreads();
    if (tid >= NC) {
        produce(st, empty, maps, t, tid & 31, L, G, e_zero, counters);
    } else {
        const LaneGeom g = lane_geom(tid);
        consume(st, empty, &cok, g, tid, L, G, reinterpret_cast<char*>(e_out), omega, counters);
    }
    __syncthreads();  // no thread leaves while boxes of this CTA may still be landing
}

bool aligned16(const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ---- host: tensor maps -----------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (fn == nullptr) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        HNS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || p == nullptr)
            fail(HNS_ERR_UNSUPPORTED, "the CUDA driver provides no cuTensorMapEncodeTiled");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// One FP16 map over `base` viewed as [num_leaves][8 x][8 y][8 z], with box (8, by, bx, 1).
void encode_map(CUtensorMap* m, const void* base, int64_t num_leaves, int bx, int by) {
    const cuuint64_t dims[4] = {8, 8, 8, (cuuint64_t)num_leaves};
    const cuuint64_t strides[3] = {16, 128, 1024};
    const cuuint32_t boxdim[4] = {8, (cuuint32_t)by, (cuuint32_t)bx, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, const_cast<void*>(base), dims, strides, boxdim,
                                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(HNS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

// Maps for (e, rhs), cached per thread for the most recent few pointer pairs: a solve alternates
// between two e buffers over one rhs, so re-encoding happens only when the arrays change.
const TensorMaps& maps_for(const void* e, const void* rhs, int64_t num_leaves) {
    struct Entry {
        const void* e = nullptr;
        const void* rhs = nullptr;
        int64_t leaves = 0;
        TensorMaps maps;
    };
    thread_local Entry cache[4];
    thread_local int next = 0;
    for (Entry& c : cache)
        if (c.e == e && c.rhs == rhs && c.leaves == num_leaves && c.leaves > 0) return c.maps;
    Entry& c = cache[next];
    next = (next + 1) % 4;
    for (int k = 0; k < kNumMaps; ++k) encode_map(&c.maps.m[k], k < kMapRFull ? e : rhs, num_leaves, kBoxX[k], kBoxY[k]);
    c.e = e, c.rhs = rhs, c.leaves = num_leaves;
    return c.maps;
}

constexpr int kGridCacheDevices = 64;

unsigned packed_grid(const Context& c) {
    static std::mutex mu;
    static int cap[kGridCacheDevices] = {};
    if (c.device < 0 || c.device >= kGridCacheDevices) fail(HNS_ERR_UNSUPPORTED, "device ordinal too large");
    int g;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cap[c.device] == 0) {
            int sms = 0, per_sm = 0;
            HNS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
            HNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbgs_packed_kernel, NT, 0));
            cap[c.device] = std::max(1, sms) * std::max(1, per_sm);
        }
        g = cap[c.device];
    }
    return (unsigned)std::min<int64_t>(g, c.topo.num_leaves);
}

}  // namespace pk

void launch_rbgs_packed_half(const Context& c, const void* rhs, const void* e_in, void* e_out, float omega,
                             const double* check, double tol2) {
    if (!pk::aligned16(rhs) || !pk::aligned16(e_in) || !pk::aligned16(e_out) || rhs == nullptr || e_out == nullptr)
        fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be non-null and 16-byte aligned");
    if (c.topo.num_leaves <= 0) return;
    // With e_in null (e = 0) the e maps are made over rhs and every e box is read at leaf -1.
    const pk::TensorMaps& maps = pk::maps_for(e_in != nullptr ? e_in : rhs, rhs, c.topo.num_leaves);
    pk::rbgs_packed_kernel<<<pk::packed_grid(c), pk::NT, 0, c.stream>>>(maps, c.topo.view, static_cast<__half*>(e_out),
                                                                       e_in == nullptr ? 1 : 0, omega, check, tol2,
                                                                       c.counters);
    HNS_LAUNCHED();
}

}  // namespace hns
