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
// Faces. A leaf's y- and z-faces are scattered over its 128-byte lines (a y-face row pair per
// x-plane, two values per z-row), and a TMA box moves whole lines, so fetching them from the
// leaf itself would move the whole leaf. Each iteration therefore also writes the faces it
// computes into a face buffer beside e (1 KiB per leaf, four 256-byte slots):
//   slot 0: rows b = 0, 1 of every x-plane    slot 1: rows b = 6, 7     (y faces, [a][2 rows])
//   slot 2: (z = 0, z = 1) of every row       slot 3: (z = 6, z = 7)    (z faces, [a][b][2])
// and the right-hand side, constant over an inner solve, is gathered once per outer step into a
// 640-byte halo record per leaf (rhs_halo_pack_kernel): its x- and y-face rows and the values
// at the leaf rows' red z-ring voxels.
//
// Staging. One producer warp stages a leaf's stencil with 21 TMA box loads (cp.async.bulk.tensor,
// no multicast): the leaf and its x-face pairs from e, the neighbours' y- and z-face slots and
// single face entries (xy edges, the ring rows' z-halo), and the leaf's right-hand side with its
// halo record. A missing neighbour is the leaf coordinate -1, which TMA fills with zeros (the
// reference's p = 0 outside the domain). Every box lands densely at a 128-byte-aligned offset.
//
// Per leaf, the update is one full iteration of redBlackGaussSeidelUpdate
// (src/Cuda/Kernel.cu:459-489) -- red on the leaf and its one-voxel face ring, then black on
// the leaf -- with the arithmetic, operation order and FP16 rounding points of
// rbgs_stream_kernel<__half> in hns_rbgs.cu, so both produce the same values to the bit (the
// tests compare them). The kernel is persistent: CTA g relaxes leaves g, g + G, ..., with
// kStages shared-memory stages; a producer warp fills them while four consumer warps relax.
//
// Work of a consumer lane: warp w owns leaf rows (a, b) with a in {2w, 2w+1}, lane =
// 16 (a - 2w) + 2 b + m, and updates the pair m (voxels 2m, 2m+1 of the colour's half-row):
//   * red: the pair from the four x/y neighbour rows and the row's own black half (one 8-byte
//     load gives all its z-neighbours), and the row's red z-ring voxel (z = 8 if a + b is even,
//     else z = -1), which only this row's black voxels need, so it stays in a register;
//   * black: the pair from the neighbour rows' updated red halves, the lane's own red pair and
//     its partner lane's (a shuffle), and the z-ring voxel; both pairs go straight to HBM, with
//     the row's z-face values and, for rows b = 0, 1, 6, 7, the row into the face buffer.
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
#include "hns_relax16.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace pk {

constexpr int NC = 96;       // consumer threads (3 warps): the relaxation
constexpr int NT = NC + 32;  // + one producer warp: the neighbour tables and the TMA boxes
constexpr int kMinBlocksPerSM = 8;
// Shared-memory stages: the producer runs up to kStages leaves ahead of the consumers.
constexpr int kStages = 4;
// Bounded mbarrier wait: give up after kWaitCycles SM cycles (about 1 s at 2 GHz); each poll
// sleeps up to kSuspendNs unless the phase completes first.
constexpr long long kWaitCycles = 2000000000LL;
constexpr uint32_t kSuspendNs = 20000;

__device__ __forceinline__ bool wait_stage(uint64_t* bar, uint32_t parity, long long max_cycles) {
    return ptx::mbar_wait_bounded_clock_sleep(bar, parity, max_cycles, kSuspendNs);
}

constexpr int kFaceBytes = kPackedFaceBytes;  // face buffer per leaf
constexpr int kHaloRows = 40;                 // rhs halo record per leaf, in 16-byte rows
constexpr int kHaloBytes = kHaloRows * 16;
static_assert(kHaloBytes == kPackedHaloBytes, "halo record size");

__host__ __device__ constexpr int nbi(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }
__host__ __device__ constexpr int parity(int a, int b) { return (a + b) & 1; }  // two's complement: ok for -1

// ---- stage layout (bytes; a row is 16 bytes = 8 packed FP16 values) -------------------------
//   E    e rows (a, b), a in [-2, 9] (12 planes of 8 rows), b in [0, 8)
//   YM   e rows (a, b), a in [0, 8), b in {-2, -1}: [a][2]     (the -y leaf's face slot 1)
//   YP   e rows (a, b), a in [0, 8), b in {8, 9}: [a][2]       (the +y leaf's face slot 0)
//   YE   e rows of the four xy-edge columns, one 128-byte slot each: (-1, {-2,-1}),
//        (8, {-2,-1}), (-1, {8,9}), (8, {8,9})                (one face entry each)
//   ZFM  (z = -2, z = -1) of rows (a, b), a, b in [0, 8)        (the -z leaf's face slot 3)
//   ZFP  (z = 8, z = 9) of rows (a, b)                          (the +z leaf's face slot 2)
//   ZX   the same pairs of the x-ring rows (a = -1, 8) at -z and +z, one 128-byte slot each
//   ZY   the z-face slots of the leaves (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1): the
//        y-ring rows' pairs are their entries (a, 7) or (a, 0)
//   B    right-hand-side rows (a, b), a, b in [0, 8)
//   RH   the leaf's rhs halo record: rows (-1, b), (8, b), (a, -1), (a, 8), then the z-ring values
constexpr int kOffE = 0;
constexpr int kOffYM = kOffE + 12 * 128;
constexpr int kOffYP = kOffYM + 256;
constexpr int kOffYE = kOffYP + 256;
constexpr int kOffZFM = kOffYE + 4 * 128;
constexpr int kOffZFP = kOffZFM + 256;
constexpr int kOffZX = kOffZFP + 256;
constexpr int kOffZY = kOffZX + 4 * 128;
constexpr int kOffB = kOffZY + 4 * 256;
constexpr int kOffRH = kOffB + 1024;
constexpr int kStageBytes = kOffRH + kHaloBytes;

// Byte offset of e row (a, b) in a stage: a in [-2, 9] for b in [0, 8); otherwise the y-face
// and edge rows listed above.
__host__ __device__ constexpr int e_row(int a, int b) {
    return (b >= 0 && b < 8) ? kOffE + (a + 2) * 128 + b * 16
           : (a >= 0 && a < 8) ? (b < 0 ? kOffYM + a * 32 + (b + 2) * 16 : kOffYP + a * 32 + (b - 8) * 16)
           : kOffYE + ((a < 0 ? 0 : 1) + (b < 0 ? 0 : 2)) * 128 + (b < 0 ? b + 2 : b - 8) * 16;
}
// Byte offset of the z-face pair of row (a, b) beyond the leaf: side 0 = (z = -2, -1) from the
// -z side, side 1 = (z = 8, 9) from the +z side. a, b in [0, 8), or one of them -1 or 8.
__host__ __device__ constexpr int z_pair(int side, int a, int b) {
    return (a >= 0 && a < 8 && b >= 0 && b < 8) ? (side ? kOffZFP : kOffZFM) + a * 32 + b * 4
           : (a < 0)  ? kOffZX + (side ? 256 : 0) + b * 4
           : (a >= 8) ? kOffZX + (side ? 384 : 128) + b * 4
           : (b < 0)  ? kOffZY + (side ? 512 : 0) + a * 32 + 7 * 4
                      : kOffZY + (side ? 768 : 256) + a * 32;
}
// Right-hand-side row (a, b): the leaf's rows, or its halo record's.
__host__ __device__ constexpr int b_row(int a, int b) {
    return (a >= 0 && a < 8 && b >= 0 && b < 8) ? kOffB + a * 128 + b * 16
           : (a < 0)  ? kOffRH + b * 16
           : (a >= 8) ? kOffRH + 128 + b * 16
           : (b < 0)  ? kOffRH + 256 + a * 16
                      : kOffRH + 384 + a * 16;
}
// Halo record, row r: r < 8: rhs row (7, r) of the -x leaf; < 16: (0, r - 8) of the +x leaf;
// < 24: (r - 16, 7) of the -y leaf; < 32: (r - 24, 0) of the +y leaf; then 64 FP16 values,
// entry a * 8 + b: the rhs at row (a, b)'s red z-ring voxel (z = 8 of the +z leaf if a + b is
// even, else z = -1 of the -z leaf).
constexpr int kHaloZ = 32 * 16;

struct __align__(128) Stage {
    uint4 data[kStageBytes / 16];
    uint64_t bar;  // completes when the stage's boxes have landed
    int nb[27];    // the staged leaf's neighbour table
};

// ---- the boxes of one leaf -------------------------------------------------------------------
// Tensor maps (one kernel parameter), all 4-D with coordinates (0, c1, c2, leaf):
enum MapId : int {
    kMapE = 0,      // e [leaf][x][y][z]: box (z 8, y 8, x 8); c1 = y, c2 = x
    kMapEXPair,     // e: box (8, 8, 2)
    kMapFace,       // face buffer [leaf][slot 4][a 8][32 bytes]: box (16, 8, 1) = a slot; c1 = a, c2 = slot
    kMapFaceEntry,  // face buffer: box (16, 1, 1) = one entry (a)
    kMapR,          // rhs [leaf][x][y][z]: box (8, 8, 8)
    kMapRH,         // rhs halo records [leaf][1][40 rows][16 bytes]: box (8, 40, 1)
    kNumMaps
};
constexpr int kMapBytes[kNumMaps] = {1024, 256, 256, 32, 1024, kHaloBytes};

struct TensorMaps {
    CUtensorMap m[kNumMaps];
};

struct Box {
    int map, c1, c2, q, dst;
};
constexpr int kBoxes = 21;

__host__ __device__ constexpr Box box(int i) {
    // clang-format off
    constexpr Box list[kBoxes] = {
        {kMapEXPair, 0, 6, nbi(-1, 0, 0), e_row(-2, 0)},     // x-face planes a = -2, -1
        {kMapE, 0, 0, nbi(0, 0, 0), e_row(0, 0)},            // the leaf
        {kMapEXPair, 0, 0, nbi(1, 0, 0), e_row(8, 0)},       // x-face planes a = 8, 9
        {kMapFace, 0, 1, nbi(0, -1, 0), kOffYM},             // y-face rows b = -2, -1
        {kMapFace, 0, 0, nbi(0, 1, 0), kOffYP},              // y-face rows b = 8, 9
        {kMapFaceEntry, 7, 1, nbi(-1, -1, 0), kOffYE},       // xy-edge columns
        {kMapFaceEntry, 0, 1, nbi(1, -1, 0), kOffYE + 128},
        {kMapFaceEntry, 7, 0, nbi(-1, 1, 0), kOffYE + 256},
        {kMapFaceEntry, 0, 0, nbi(1, 1, 0), kOffYE + 384},
        {kMapFace, 0, 3, nbi(0, 0, -1), kOffZFM},            // z faces
        {kMapFace, 0, 2, nbi(0, 0, 1), kOffZFP},
        {kMapFaceEntry, 7, 3, nbi(-1, 0, -1), kOffZX},       // x-ring rows' z-halo
        {kMapFaceEntry, 0, 3, nbi(1, 0, -1), kOffZX + 128},
        {kMapFaceEntry, 7, 2, nbi(-1, 0, 1), kOffZX + 256},
        {kMapFaceEntry, 0, 2, nbi(1, 0, 1), kOffZX + 384},
        {kMapFace, 0, 3, nbi(0, -1, -1), kOffZY},            // y-ring rows' z-halo
        {kMapFace, 0, 3, nbi(0, 1, -1), kOffZY + 256},
        {kMapFace, 0, 2, nbi(0, -1, 1), kOffZY + 512},
        {kMapFace, 0, 2, nbi(0, 1, 1), kOffZY + 768},
        {kMapR, 0, 0, nbi(0, 0, 0), kOffB},                  // right-hand side
        {kMapRH, 0, 0, nbi(0, 0, 0), kOffRH},                // its halo record
    };
    // clang-format on
    return list[i];
}

constexpr int stage_tx_bytes() {
    int s = 0;
    for (int i = 0; i < kBoxes; ++i) s += kMapBytes[box(i).map];
    return s;
}
constexpr uint32_t kStageTx = stage_tx_bytes();

// Fixed shared-memory byte offsets (relative to a stage) of one consumer thread's loads, and
// its offsets in a leaf's output blocks. Warps 0 and 1: leaf row (a, b) = (4 w + lane / 8,
// lane % 8), all four red then all four black voxels; warp 2: ring row lane (lanes 0-15 the
// x-ring rows (-1, b), (8, b); 16-31 the y-ring rows (a, -1), (a, 8)), its four red voxels.
struct LaneGeom {
    int a, b, pi;  // the row and the parity of a + b
    int red;       // the row's red half (8 bytes)
    int xp, xm;    // the x-neighbour rows' halves at the red positions (leaf rows: red +- 128)
    int yp, ym;    // the y-neighbour rows' halves at the red positions
    int dk;        // black half - red half (8 - 16 pi)
    int b_red;     // right-hand side of the red half; the black half's at + dk
    int zlo;       // z = -1 of the row; z = 8 at + kZHi (leaf rows); for ring rows the z-halo
                   // their red voxels need: z = -1 if pi = 0, else z = 8
    int zc;        // the row's red z-ring voxel (z = 8 if pi = 0, else z = -1)
    int zxp, zxm, zyp, zym;  // its x and y neighbours
    int zfar;      // its z-neighbour beyond: z = 9 if pi = 0, else z = -2
    int bz;        // right-hand side of the z-ring voxel
    int zq;        // neighbour-table index of the leaf holding the z-ring voxel
    int q;         // ring rows: neighbour-table index of the row's leaf
    int gout;      // byte offset of the row in a leaf's 1 KiB block of e
    int zface;     // byte offset of the row's (z0, z1) pair in a leaf's face block; (z6, z7) at + 256
    int yface;     // byte offset of the row in the face block (rows b = 0, 1, 6, 7), else -1
};
constexpr int kZHi = z_pair(1, 0, 0) - (z_pair(0, 0, 0) + 2);

__host__ __device__ inline LaneGeom lane_geom(int tid) {
    LaneGeom g{};
    const int lane = tid & 31, warp = tid >> 5;
    if (warp < 2) {
        g.a = 4 * warp + (lane >> 3);
        g.b = lane & 7;
    } else if (lane < 16) {
        g.a = (lane >> 3) ? 8 : -1, g.b = lane & 7;
        g.q = nbi((lane >> 3) ? 1 : -1, 0, 0);
    } else {
        g.a = lane & 7, g.b = ((lane >> 3) & 1) ? 8 : -1;
        g.q = nbi(0, ((lane >> 3) & 1) ? 1 : -1, 0);
    }
    g.pi = parity(g.a, g.b);
    const int pos = 8 * g.pi;
    g.red = e_row(g.a, g.b) + pos;
    g.xp = e_row(g.a + 1, g.b) + pos;
    g.xm = e_row(g.a - 1, g.b) + pos;
    g.yp = e_row(g.a, g.b + 1) + pos;
    g.ym = e_row(g.a, g.b - 1) + pos;
    g.dk = 8 - 16 * g.pi;
    g.b_red = b_row(g.a, g.b) + pos;
    if (warp < 2) {
        g.zlo = z_pair(0, g.a, g.b) + 2;
        const int side = g.pi ? 0 : 1, zpos = g.pi ? 2 : 0;
        g.zc = z_pair(side, g.a, g.b) + zpos;
        g.zxp = z_pair(side, g.a + 1, g.b) + zpos;
        g.zxm = z_pair(side, g.a - 1, g.b) + zpos;
        g.zyp = z_pair(side, g.a, g.b + 1) + zpos;
        g.zym = z_pair(side, g.a, g.b - 1) + zpos;
        g.zfar = g.pi ? g.zc - 2 : g.zc + 2;
        g.bz = kOffRH + kHaloZ + (g.a * 8 + g.b) * 2;
        g.zq = nbi(0, 0, g.pi ? -1 : 1);
        g.gout = (g.a * 64 + g.b * 8) * 2;
        g.zface = 2 * 256 + g.a * 32 + g.b * 4;
        g.yface = g.b < 2 ? g.a * 32 + g.b * 16 : g.b >= 6 ? 256 + g.a * 32 + (g.b - 6) * 16 : -1;
    } else {
        g.zlo = g.pi ? z_pair(1, g.a, g.b) : z_pair(0, g.a, g.b) + 2;
    }
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

using namespace relax16;

// Issues the boxes of the leaf whose neighbour table is in S.nb into stage S (one thread).
// e_zero: e = 0 (the first iteration of a solve), so every box of e or its faces is read at
// leaf -1 and arrives as zeros.
__device__ __forceinline__ void stage_issue(Stage& S, const TensorMaps& maps, int e_zero) {
    const uint32_t base = ptx::smem_addr(&S);
    ptx::mbar_arrive_expect_tx(&S.bar, kStageTx);
#pragma unroll
    for (int i = 0; i < kBoxes; ++i) {
        const Box bx = box(i);
        const int leaf = (e_zero && bx.map < kMapR) ? -1 : S.nb[bx.q];
        ptx::tma_load_4d(base + bx.dst, &maps.m[bx.map], 0, bx.c1, bx.c2, leaf, &S.bar);
    }
}

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"r"(NC) : "memory"); }

// The z-neighbour pairs of a row's four red voxels (pairs 0-1 and 2-3) from its black half
// (k01, k23) and its values beyond the leaf at z = -1 (zlo) and z = 8 (zhi): with pi = 0 the
// red voxels are at even z, their z+ the black values at the same index and their z- one
// index lower; with pi = 1 the other way round.
__device__ __forceinline__ void red_z(uint32_t k01, uint32_t k23, uint32_t zlo, uint32_t zhi, int pi, uint32_t& zp0,
                                      uint32_t& zp1, uint32_t& zm0, uint32_t& zm1) {
    const uint32_t mid = __byte_perm(k01, k23, 0x5432);  // black values 1, 2
    if (pi == 0) {
        zp0 = k01, zp1 = k23;
        zm0 = __byte_perm(zlo, k01, 0x5410), zm1 = mid;  // (z = -1, 0), (1, 2)
    } else {
        zm0 = k01, zm1 = k23;
        zp0 = mid, zp1 = __byte_perm(k23, zhi, 0x5432);  // (1, 2), (3, z = 8)
    }
}

__device__ __forceinline__ void sts64(uint32_t a, uint32_t lo, uint32_t hi) {
    asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(a), "r"(lo), "r"(hi));
}

// Consumers (warps 0-2): relax the CTA's leaves in order from the staged boxes.
__device__ __forceinline__ void consume(Stage* st, uint64_t* empty, int* cok, const LaneGeom& g, int tid, int64_t L,
                                        int64_t G, char* out, char* faces, float omega,
                                        unsigned long long* counters) {
    const int warp = tid >> 5, lane = tid & 31;
    int64_t leaf = blockIdx.x;
    for (uint32_t j = 0; leaf < L; ++j, leaf += G) {
        const int s = j % kStages;
        Stage& cur = st[s];
        // One thread waits for the stage's boxes; the others wait at the consumer barrier, and
        // all of them read the outcome after it.
        if (tid == 0) {
            const bool landed = wait_stage(&cur.bar, (j / kStages) & 1, kWaitCycles);
            if (!landed && counters != nullptr) atomicExch(counters + 1, 1ull);
            *cok = landed ? 1 : 0;
        }
        consumer_sync();
        if (!*cok) return;  // e_out keeps its old values for the leaves left
        const uint32_t S = ptx::smem_addr(&cur);

        // ---- red: the row's four red voxels, as two pairs ----
        uint32_t k01, k23, c01, c23, xp0, xp1, xm0, xm1, yp0, yp1, ym0, ym1, b01, b23;
        lds64(S + g.red + g.dk, k01, k23);  // the row's black half
        lds64(S + g.red, c01, c23);
        lds64(S + g.xp, xp0, xp1);
        lds64(S + g.xm, xm0, xm1);
        lds64(S + g.yp, yp0, yp1);
        lds64(S + g.ym, ym0, ym1);
        lds64(S + g.b_red, b01, b23);
        const bool leaf_row = warp < 2;
        const uint32_t zlo = lds16(S + g.zlo), zhi = leaf_row ? lds16(S + g.zlo + kZHi) : zlo;
        uint32_t zp0, zp1, zm0, zm1;
        red_z(k01, k23, zlo, zhi, g.pi, zp0, zp1, zm0, zm1);
        const uint32_t r01 = relax2(xp0, xm0, yp0, ym0, zp0, zm0, b01, c01, omega);
        const uint32_t r23 = relax2(xp1, xm1, yp1, ym1, zp1, zm1, b23, c23, omega);
        uint32_t zring = 0;
        if (leaf_row) {
            sts64(S + g.red, r01, r23);
            // The row's red z-ring voxel: its x/y neighbours are the neighbour rows' values at
            // the same z; its z-neighbours are the row's black value at z = 7 (pi = 0) or z = 0
            // (pi = 1) and the value beyond it.
            const uint32_t near = g.pi ? (k01 & 0xffffu) : (k23 >> 16);
            const uint32_t far = lds16(S + g.zfar);
            const uint32_t ctr = g.pi ? zlo : zhi;
            const float v = relax1(lds16(S + g.zxp), lds16(S + g.zxm), lds16(S + g.zyp), lds16(S + g.zym),
                                   g.pi ? near : far, g.pi ? far : near, lds16(S + g.bz), ctr, omega);
            zring = cur.nb[g.zq] >= 0 ? round_half(v) : ctr;
        } else if (cur.nb[g.q] >= 0) {  // ring row of an existing neighbour leaf
            sts64(S + g.red, r01, r23);
        }
        consumer_sync();

        if (leaf_row) {
            // ---- black: the row's four black voxels ----
            // z-neighbours from the row's updated red values r0..r3 and the z-ring voxel:
            // pi = 0 (black at odd z): z- = r[i], z+ = r[i+1] (r[4] = z-ring at z = 8);
            // pi = 1 (black at even z): z+ = r[i], z- = r[i-1] (r[-1] = z-ring at z = -1).
            const uint32_t mid = __byte_perm(r01, r23, 0x5432);  // r1, r2
            uint32_t bzp0, bzp1, bzm0, bzm1;
            if (g.pi == 0) {
                bzm0 = r01, bzm1 = r23;
                bzp0 = mid, bzp1 = __byte_perm(r23, zring, 0x5432);
            } else {
                bzp0 = r01, bzp1 = r23;
                bzm0 = __byte_perm(zring, r01, 0x5410), bzm1 = mid;
            }
            const uint32_t ob = S + g.red + g.dk;
            lds64(ob + 128, xp0, xp1);
            lds64(ob - 128, xm0, xm1);
            lds64(S + g.yp + g.dk, yp0, yp1);
            lds64(S + g.ym + g.dk, ym0, ym1);
            lds64(S + g.b_red + g.dk, b01, b23);
            const uint32_t k01n = relax2(xp0, xm0, yp0, ym0, bzp0, bzm0, b01, k01, omega);
            const uint32_t k23n = relax2(xp1, xm1, yp1, ym1, bzp1, bzm1, b23, k23, omega);
            // The row (even-z half first) into e_out, its z-face pairs (z0, z1) and (z6, z7),
            // and on the y faces the row into the face buffer.
            const uint32_t e01 = g.pi ? k01n : r01, e23 = g.pi ? k23n : r23;
            const uint32_t o01 = g.pi ? r01 : k01n, o23 = g.pi ? r23 : k23n;
            const uint4 rowv = make_uint4(e01, e23, o01, o23);
            *reinterpret_cast<uint4*>(out + (leaf << 10) + g.gout) = rowv;
            char* face = faces + (leaf << 10);
            *reinterpret_cast<uint32_t*>(face + g.zface) = __byte_perm(e01, o01, 0x5410);        // (z0, z1)
            *reinterpret_cast<uint32_t*>(face + g.zface + 256) = __byte_perm(e23, o23, 0x7632);  // (z6, z7)
            if (g.yface >= 0) *reinterpret_cast<uint4*>(face + g.yface) = rowv;
        }
        // This warp is done with the stage: order its reads and writes of it before the next
        // boxes (async proxy) and release it to the producer.
        ptx::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) ptx::mbar_arrive(&empty[s]);
    }
}

// Producer (warp 3): for each of the CTA's leaves, waits until the consumers have released the
// stage's previous leaf, writes the leaf's neighbour table into it and issues its boxes. If a
// release never comes (the consumers stopped), it waits for its boxes still in flight so that
// none lands after the CTA has exited.
__device__ __forceinline__ void produce(Stage* st, uint64_t* empty, const TensorMaps& maps, const TopoView& t,
                                        int lane, int64_t L, int64_t G, int e_zero, unsigned long long* counters) {
    int64_t leaf = blockIdx.x;
    int nb_next = (lane < 27 && leaf < L) ? __ldg(t.nbr27 + leaf * 27 + lane) : -1;
    for (uint32_t j = 0; leaf < L; ++j, leaf += G) {
        const int s = j % kStages;
        const int nb = nb_next;
        nb_next = (lane < 27 && leaf + G < L) ? __ldg(t.nbr27 + (leaf + G) * 27 + lane) : -1;
        bool released = true;
        if (j >= kStages && lane == 0) released = wait_stage(&empty[s], (j / kStages - 1) & 1, kWaitCycles);
        released = __shfl_sync(0xffffffffu, released ? 1 : 0, 0) != 0;
        if (!released) {
            if (lane == 0) {
                if (counters != nullptr) atomicExch(counters + 1, 1ull);
                for (uint32_t k = j > kStages ? j - kStages : 0; k < j; ++k)
                    (void)wait_stage(&st[k % kStages].bar, (k / kStages) & 1, kWaitCycles);
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
    rbgs_packed_kernel(const __grid_constant__ TensorMaps maps, TopoView t, __half* __restrict__ e_out,
                       char* __restrict__ faces_out, int e_zero, float omega, const double* __restrict__ check,
                       double tol2, unsigned long long* __restrict__ counters) {
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
        consume(st, empty, &cok, g, tid, L, G, reinterpret_cast<char*>(e_out), faces_out, omega, counters);
    }
    __syncthreads();  // no thread leaves while boxes of this CTA may still be landing
}

// The rhs halo records of every leaf (layout at kHaloRows): block = leaf, threads 0-31 copy the
// 32 face rows, threads 32-95 the 64 z-ring values. Rows and values of missing leaves are 0.
__global__ void __launch_bounds__(96) rhs_halo_pack_kernel(TopoView t, const __half* __restrict__ rhs,
                                                             uint4* __restrict__ halo, const double* __restrict__ check,
                                                             double tol2) {
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int64_t leaf = blockIdx.x;
    const int tid = threadIdx.x;
    const int* nb = t.nbr27 + leaf * 27;
    uint4* out = halo + leaf * kHaloRows;
    const uint4* r4 = reinterpret_cast<const uint4*>(rhs);  // row (l, a, b) at r4[l * 64 + a * 8 + b]
    if (tid < 32) {
        const int k = tid & 7, part = tid >> 3;
        const int q = part == 0 ? nbi(-1, 0, 0) : part == 1 ? nbi(1, 0, 0) : part == 2 ? nbi(0, -1, 0) : nbi(0, 1, 0);
        const int a = part == 0 ? 7 : part == 1 ? 0 : k, b = part < 2 ? k : part == 2 ? 7 : 0;
        const int l = __ldg(nb + q);
        out[tid] = l >= 0 ? __ldg(r4 + (int64_t)l * 64 + a * 8 + b) : make_uint4(0, 0, 0, 0);
    } else {
        const int e = tid - 32, a = e >> 3, b = e & 7, even = parity(a, b) == 0;
        const int l = __ldg(nb + nbi(0, 0, even ? 1 : -1));
        // z = 0 of the +z leaf's row is at packed position 0, z = 7 of the -z leaf's at 7.
        const __half v = l >= 0 ? rhs[((int64_t)l * 64 + a * 8 + b) * 8 + (even ? 0 : 7)] : __ushort_as_half(0);
        reinterpret_cast<__half*>(out + 32)[e] = v;
    }
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

// A 4-D FP16 map over `base` (dims innermost first, strides in bytes of dims 1-3) with a box.
void encode4(CUtensorMap* m, const void* base, const cuuint64_t (&dims)[4], const cuuint64_t (&strides)[3],
             const cuuint32_t (&boxdim)[4]) {
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, const_cast<void*>(base), dims, strides, boxdim,
                                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(HNS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

void encode_maps(TensorMaps& t, const void* e, const void* faces, const void* rhs, const void* halo, int64_t L) {
    const cuuint64_t leaf_dims[4] = {8, 8, 8, (cuuint64_t)L}, leaf_str[3] = {16, 128, 1024};
    const cuuint64_t face_dims[4] = {16, 8, 4, (cuuint64_t)L}, face_str[3] = {32, 256, (cuuint64_t)kFaceBytes};
    const cuuint64_t halo_dims[4] = {8, kHaloRows, 1, (cuuint64_t)L}, halo_str[3] = {16, kHaloBytes, kHaloBytes};
    encode4(&t.m[kMapE], e, leaf_dims, leaf_str, {8, 8, 8, 1});
    encode4(&t.m[kMapEXPair], e, leaf_dims, leaf_str, {8, 8, 2, 1});
    encode4(&t.m[kMapFace], faces, face_dims, face_str, {16, 8, 1, 1});
    encode4(&t.m[kMapFaceEntry], faces, face_dims, face_str, {16, 1, 1, 1});
    encode4(&t.m[kMapR], rhs, leaf_dims, leaf_str, {8, 8, 8, 1});
    encode4(&t.m[kMapRH], halo, halo_dims, halo_str, {8, kHaloRows, 1, 1});
}

// Maps for (e, faces, rhs, halo), cached per thread for the most recent few combinations: a solve
// alternates between two e buffers over one rhs, so re-encoding happens only when arrays change.
const TensorMaps& maps_for(const void* e, const void* faces, const void* rhs, const void* halo, int64_t L) {
    struct Entry {
        const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
        int64_t leaves = 0;
        TensorMaps maps;
    };
    thread_local Entry cache[4];
    thread_local int next = 0;
    for (Entry& c : cache)
        if (c.leaves == L && c.key[0] == e && c.key[1] == faces && c.key[2] == rhs && c.key[3] == halo) return c.maps;
    Entry& c = cache[next];
    next = (next + 1) % 4;
    encode_maps(c.maps, e, faces, rhs, halo, L);
    c.key[0] = e, c.key[1] = faces, c.key[2] = rhs, c.key[3] = halo, c.leaves = L;
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

void launch_rhs_halo_pack(const Context& c, const void* rhs, void* halo, const double* check, double tol2) {
    if (!pk::aligned16(rhs) || !pk::aligned16(halo) || rhs == nullptr || halo == nullptr)
        fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be non-null and 16-byte aligned");
    if (c.topo.num_leaves <= 0) return;
    pk::rhs_halo_pack_kernel<<<(unsigned)c.topo.num_leaves, 96, 0, c.stream>>>(
        c.topo.view, static_cast<const __half*>(rhs), static_cast<uint4*>(halo), check, tol2);
    HNS_LAUNCHED();
}

void launch_rbgs_packed_half(const Context& c, const void* rhs, const void* halo, const void* e_in, const void* faces_in,
                             void* e_out, void* faces_out, float omega, const double* check, double tol2) {
    const void* ptrs[6] = {rhs, halo, e_in, faces_in, e_out, faces_out};
    for (int k = 0; k < 6; ++k)
        if (!pk::aligned16(ptrs[k]) || (ptrs[k] == nullptr && k != 2 && k != 3))
            fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be 16-byte aligned (only e_in and its faces may be null)");
    if (c.topo.num_leaves <= 0) return;
    // With e_in null (e = 0) the maps of e and its faces are made over arrays of the same shapes
    // (rhs, faces_out) and every box of them is read at leaf -1, so no memory is read.
    const bool zero = e_in == nullptr || faces_in == nullptr;
    const pk::TensorMaps& maps = pk::maps_for(zero ? rhs : e_in, zero ? faces_out : faces_in, rhs, halo, c.topo.num_leaves);
    pk::rbgs_packed_kernel<<<pk::packed_grid(c), pk::NT, 0, c.stream>>>(maps, c.topo.view, static_cast<__half*>(e_out),
                                                                       static_cast<char*>(faces_out), zero ? 1 : 0,
                                                                       omega, check, tol2, c.counters);
    HNS_LAUNCHED();
}

}  // namespace hns
