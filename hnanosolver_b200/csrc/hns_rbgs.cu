// The red-black SOR iteration, staged with asynchronous copies and relaxed row by row.
//
// A persistent kernel: each 128-thread CTA relaxes a sequence of 8^3 leaves, one full
// iteration of redBlackGaussSeidelUpdate (src/Cuda/Kernel.cu:459-489) per leaf -- red on the
// leaf and its one-voxel face ring, then black on the leaf -- from p_in to p_out, reading p
// with a two-voxel halo and the right-hand side with a one-voxel halo, as
// rbgs_iteration_kernel in hns_kernels.cu does (same arithmetic, same results to the bit).
// How the stencil reaches shared memory and is computed:
//
//   * Shared memory holds z-rows of 8 values. A leaf's slot order is x-major
//     (x*64 + y*8 + z), so every x-plane of a leaf (64 values), every pair of y-rows of a
//     plane (16 values) and every single row (8 values) is contiguous in HBM and lands
//     contiguously in the row layout: 58 pieces (8 interior planes, x-face planes, y-face
//     rows, xy-edge rows of p and of the right-hand side) are fetched by cp.async.bulk,
//     issued by one warp. A piece whose leaf does not exist is copied from a page of zeros.
//   * The z-halo (values at z = -2, -1, 8, 9 of a row) is a pair of values per row in HBM;
//     every thread fetches its pairs with cp.async, counted on the same mbarrier.
//   * Two stages: the copies of the CTA's next leaf are in flight while the current one is
//     relaxed, so the copy latency is hidden behind the arithmetic.
//   * Voxels are relaxed one per lane in warp tasks of 32 whose shared-memory reads hit 32
//     different banks. Red: the leaf's 256, the x/y ring's 128 and the z ring's 64; black:
//     the leaf's 256.
//
// T is the storage type of p and the right-hand side (float, or __half for the inner solve
// of the mixed-precision refinement); arithmetic is FP32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "hns_internal.cuh"
#include "hns_ptx.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

constexpr int NT = 128;
constexpr int kMinBlocksPerSM = 8;
// Bounded mbarrier wait: at most kMaxPolls polls of at most kSuspendNs each -- far above
// any real copy latency (microseconds), and about 1 s when every poll sleeps its full hint.
constexpr uint32_t kSuspendNs = 20000;
constexpr uint32_t kMaxPolls = 50000;

// 2 KiB of zeros: the source of every staged piece whose leaf does not exist (and of p when
// the iteration starts from p = 0), so that every copy is unconditional.
__device__ __align__(128) float g_zero_leaf[512];

// Neighbour-table index of the leaf at offset (dx, dy, dz) in {-1,0,1}^3.
__host__ __device__ constexpr int nbi(int dx, int dy, int dz) { return (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1); }

// A stage is one leaf's stencil in shared memory, as one array of T with four regions:
//   P  [kOffP,  +1152): p rows (a+2, b+2) for a, b in [-2, 9], z in [0, 8)
//   B  [kOffB,  +800):  right-hand-side rows (a+1, b+1) for a, b in [-1, 8]
//   PZ [kOffPZ, +576):  p at z = -2, -1, 8, 9 of row (a+2, b+2)
//   BZ [kOffBZ, +256):  right-hand side at z = -2, -1, 8, 9 of leaf row (a, b) (-1 and 8 used)
constexpr int kOffP = 0;
constexpr int kOffB = kOffP + 12 * 12 * 8;
constexpr int kOffPZ = kOffB + 10 * 10 * 8;
constexpr int kOffBZ = kOffPZ + 12 * 12 * 4;
constexpr int kStageValues = kOffBZ + 8 * 8 * 4;
// Values a stage receives in 16-byte chunks: per interior plane a in [0, 8) the p and rhs
// planes (64 + 64), the p y-face row pairs (16 + 16) and the rhs y-face rows (8 + 8); four p
// x-face planes, two rhs x-face planes, four p xy-edge rows. Plus 320 z-halo pairs.
constexpr int kStagedValues = 8 * (64 + 64 + 16 + 16 + 8 + 8) + 4 * 64 + 2 * 64 + 4 * 8;
constexpr int kHaloPairs = 320;

template <typename T>
struct __align__(128) Stage {
    T v[kStageValues];
    const char* src[54];  // leaf base of neighbour q (q < 27: p, else rhs of q - 27), or the zero page
    uint64_t bar;         // completes when every thread's copies into this stage have landed
    int nb[27];           // the staged leaf's neighbour table
};

__host__ __device__ constexpr int prow(int a, int b) { return (a + 2) * 12 + (b + 2); }
__host__ __device__ constexpr int brow(int a, int b) { return (a + 1) * 10 + (b + 1); }

// One staging copy, packed: source table index (bits 0-5, into Stage::src), byte offset in
// the source leaf (bits 6-16), byte offset in the stage (bits 17-31).
__host__ __device__ constexpr uint32_t copy_desc(int q, int src_bytes, int dst_bytes) {
    return (uint32_t)q | ((uint32_t)src_bytes << 6) | ((uint32_t)dst_bytes << 17);
}

// Every copy that stages a leaf, for values of S bytes: the 16-byte chunks of the pieces
// listed at kStagedValues, then the z-halo pairs -- z = 6,7 of the -z leaf's row or z = 0,1 of
// the +z leaf's row, for p (leaf rows), the right-hand side (leaf rows) and p (x/y ring rows,
// from the edge leaves). Built at compile time.
template <int S>
struct CopyTable {
    static constexpr int kChunkValues = 16 / S;
    static constexpr int kChunks = kStagedValues / kChunkValues;
    uint32_t chunk[kChunks];
    uint32_t pair[kHaloPairs];
    int n;
    constexpr void piece(int q, int src, int dst, int count) {
        for (int i = 0; i < count; i += kChunkValues) chunk[n++] = copy_desc(q, (src + i) * S, (dst + i) * S);
    }
};

template <int S>
constexpr CopyTable<S> make_copy_table() {
    CopyTable<S> t{};
    t.n = 0;
    const int self = nbi(0, 0, 0), my = nbi(0, -1, 0), py = nbi(0, 1, 0);
    for (int a = 0; a < 8; ++a) {
        t.piece(self, a * 64, kOffP + prow(a, 0) * 8, 64);
        t.piece(27 + self, a * 64, kOffB + brow(a, 0) * 8, 64);
        t.piece(my, a * 64 + 48, kOffP + prow(a, -2) * 8, 16);
        t.piece(py, a * 64, kOffP + prow(a, 8) * 8, 16);
        t.piece(27 + my, a * 64 + 56, kOffB + brow(a, -1) * 8, 8);
        t.piece(27 + py, a * 64, kOffB + brow(a, 8) * 8, 8);
    }
    for (int q = 0; q < 4; ++q) {  // p x-face planes a = -2, -1, 8, 9
        const int a = q < 2 ? q - 2 : q + 6;
        t.piece(nbi(a < 0 ? -1 : 1, 0, 0), (a & 7) * 64, kOffP + prow(a, 0) * 8, 64);
    }
    for (int q = 0; q < 2; ++q) {  // rhs x-face planes a = -1, 8
        const int a = q == 0 ? -1 : 8;
        t.piece(27 + nbi(a < 0 ? -1 : 1, 0, 0), (a & 7) * 64, kOffB + brow(a, 0) * 8, 64);
    }
    for (int q = 0; q < 4; ++q) {  // p xy-edge rows (a, b) in {-1, 8}^2
        const int a = (q & 2) ? 8 : -1, b = (q & 1) ? 8 : -1;
        t.piece(nbi(a < 0 ? -1 : 1, b < 0 ? -1 : 1, 0), (a & 7) * 64 + (b & 7) * 8, kOffP + prow(a, b) * 8, 8);
    }
    for (int j = 0; j < 128; ++j) {  // leaf rows: (a, b) = ((j & 63) >> 3, j & 7), side j >> 6
        const int hi = j >> 6, row = j & 63, a = row >> 3, b = row & 7, q = nbi(0, 0, hi ? 1 : -1);
        const int src = (a * 64 + b * 8 + (hi ? 0 : 6)) * S;
        t.pair[j] = copy_desc(q, src, (kOffPZ + prow(a, b) * 4 + (hi ? 2 : 0)) * S);
        t.pair[128 + j] = copy_desc(27 + q, src, (kOffBZ + row * 4 + (hi ? 2 : 0)) * S);
    }
    for (int v = 0; v < 64; ++v) {  // x/y ring rows, z = -1 / 8, from the edge leaves
        const int side = v >> 4, zhi = (v >> 3) & 1, k = v & 7;
        const int a = side == 0 ? -1 : side == 1 ? 8 : k, b = side == 2 ? -1 : side == 3 ? 8 : k;
        const int la = side == 0 ? -1 : side == 1 ? 1 : 0, lb = side == 2 ? -1 : side == 3 ? 1 : 0;
        t.pair[256 + v] = copy_desc(nbi(la, lb, zhi ? 1 : -1), ((a & 7) * 64 + (b & 7) * 8 + (zhi ? 0 : 6)) * S,
                                    (kOffPZ + prow(a, b) * 4 + (zhi ? 2 : 0)) * S);
    }
    return t;
}

__device__ const CopyTable<4> g_copies4 = make_copy_table<4>();
__device__ const CopyTable<2> g_copies2 = make_copy_table<2>();

template <typename T>
__device__ __forceinline__ const CopyTable<sizeof(T)>& copy_table();
template <>
__device__ __forceinline__ const CopyTable<4>& copy_table<float>() { return g_copies4; }
template <>
__device__ __forceinline__ const CopyTable<2>& copy_table<__half>() { return g_copies2; }

// A thread's share of the copies: chunk slot k is chunk 128 k + tid (the last, partial slot
// counts down from tid 127 so that its copies fall on the threads without a ring pair); pair
// slots 0 and 1 are pairs tid and 128 + tid, slot 2 the ring pair 256 + tid for tid < 64.
template <typename T>
struct CopyPlan {
    static constexpr int kChunks = CopyTable<sizeof(T)>::kChunks;
    static constexpr int kSlots = (kChunks + NT - 1) / NT;
    static constexpr int kLastCount = kChunks - (kSlots - 1) * NT;
    uint32_t chunk[kSlots];
    uint32_t pair[3];
    bool last;  // this thread has a chunk in the partial last slot
};

template <typename T>
__device__ __forceinline__ CopyPlan<T> copy_plan(int tid) {
    using P = CopyPlan<T>;
    const CopyTable<sizeof(T)>& t = copy_table<T>();
    P p;
#pragma unroll
    for (int k = 0; k < P::kSlots - 1; ++k) p.chunk[k] = t.chunk[k * NT + tid];
    p.last = (NT - 1 - tid) < P::kLastCount;
    p.chunk[P::kSlots - 1] = p.last ? t.chunk[(P::kSlots - 1) * NT + (NT - 1 - tid)] : 0u;
    p.pair[0] = t.pair[tid];
    p.pair[1] = t.pair[128 + tid];
    p.pair[2] = tid < 64 ? t.pair[256 + tid] : 0u;
    return p;
}

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

// One SOR update, as offsets into a stage: the voxel c, its z+ and z- neighbours and its
// right-hand side; the x and y neighbours are at c +- SX and c +- SY.
struct Cell {
    int c, zp, zm, b;
};

// Voxel (a, b, d), d in [0, 8), of a row staged in P (the leaf's rows, the x and y ring rows).
__device__ __forceinline__ Cell row_cell(int a, int b, int d) {
    const int r = prow(a, b), c = kOffP + r * 8 + d;
    return {c, d < 7 ? c + 1 : kOffPZ + r * 4 + 2, d > 0 ? c - 1 : kOffPZ + r * 4 + 1, kOffB + brow(a, b) * 8 + d};
}

// z-ring voxel (a, b, -1) (hi = 0) or (a, b, 8) (hi = 1) of leaf row (a, b): it and its x/y
// neighbours live in PZ (x +- 48, y +- 4).
__device__ __forceinline__ Cell zring_cell(int a, int b, int hi) {
    const int r = prow(a, b), k = hi ? 2 : 1;
    return {kOffPZ + r * 4 + k, hi ? kOffPZ + r * 4 + 3 : kOffP + r * 8, hi ? kOffP + r * 8 + 7 : kOffPZ + r * 4,
            kOffBZ + (a * 8 + b) * 4 + k};
}

// The update of redBlackGaussSeidelUpdate (src/Cuda/Kernel.cu:459-489) with the six-neighbour
// sum in the reference's order (x+, x-, y+, y-, z+, z-).
template <int SX, int SY, typename T>
__device__ __forceinline__ void relax(T* v, const Cell& o, float dx2, float omega) {
    const float sum = to_f(v[o.c + SX]) + to_f(v[o.c - SX]) + to_f(v[o.c + SY]) + to_f(v[o.c - SY]) + to_f(v[o.zp]) +
                      to_f(v[o.zm]);
    const float pgs = (sum - to_f(v[o.b]) * dx2) * dev::kInv6;
    const float po = to_f(v[o.c]);
    v[o.c] = from_f<T>(po + omega * (pgs - po));
}

// Value of p (pv) and of the right-hand side (bv) at local (a, b, d), d in [-1, 8] (residual).
template <typename T>
__device__ __forceinline__ float pv(const T* v, int a, int b, int d) {
    const int r = prow(a, b);
    if ((unsigned)d < 8u) return to_f(v[kOffP + r * 8 + d]);
    return to_f(v[kOffPZ + r * 4 + (d < 0 ? d + 2 : d - 6)]);
}

template <typename T>
__device__ __forceinline__ float bv(const T* v, int a, int b, int d) {
    if ((unsigned)d < 8u) return to_f(v[kOffB + brow(a, b) * 8 + d]);
    return to_f(v[kOffBZ + (a * 8 + b) * 4 + (d < 0 ? 1 : 2)]);
}

template <typename T>
__device__ __forceinline__ const char* leaf_src(const T* a, int l, const T* zero) {
    return reinterpret_cast<const char*>((a != nullptr && l >= 0) ? a + ((int64_t)l << 9) : zero);
}

// Starts every copy of a leaf's stencil into stage S (whose source table is filled in): each
// thread issues its chunks and pairs with cp.async and arrives on S.bar when they have landed
// (the barrier expects one arrival per thread).
template <typename T>
__device__ __forceinline__ void stage_issue(Stage<T>& S, const CopyPlan<T>& cp, int tid) {
    using P = CopyPlan<T>;
    const uint32_t base = ptx::smem_addr(&S);
#pragma unroll
    for (int k = 0; k < P::kSlots; ++k) {
        if (k < P::kSlots - 1 || cp.last) {
            const uint32_t d = cp.chunk[k];
            ptx::cp_async_cg16(base + (d >> 17), S.src[d & 63] + ((d >> 6) & 2047));
        }
    }
    constexpr int kPair = 2 * (int)sizeof(T);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k < 2 || tid < 64) {
            const uint32_t d = cp.pair[k];
            ptx::cp_async_ca<kPair>(base + (d >> 17), S.src[d & 63] + ((d >> 6) & 2047));
        }
    }
    ptx::cp_async_mbar_arrive_noinc(&S.bar);
}

// Persistent red-black SOR iteration: CTA g relaxes leaves g, g + G, g + 2G, ... (G = grid
// size), each one full iteration of redBlackGaussSeidelUpdate (src/Cuda/Kernel.cu:459-489) --
// red on the leaf and its one-voxel face ring, then black on the leaf -- from p_in to p_out.
// Two stages: while leaf i is relaxed, the copies of leaf i+1 are in flight, and the
// neighbour table of leaf i+2 is being loaded.
//
// Warp w relaxes, per leaf, the red warp tasks w, w+4, w+8 (and w+12 for w < 2) and the black
// tasks w and w+4. A task is 32 voxels of one colour, one per lane, whose shared-memory reads
// fall in 32 different banks: 4 consecutive y-rows of two x-rows 12 rows apart (the same bank
// base) whose voxels of the colour have opposite parity in z, 4 voxels per row. Tasks 0-7 are
// the leaf's rows; 8-9 the x-ring rows, 10-11 the y-ring rows, 12-13 the z-ring voxels (red
// only). Every offset is fixed per thread and computed once.
template <typename T>
__global__ void __launch_bounds__(NT, kMinBlocksPerSM)
    rbgs_stream_kernel(TopoView t, const T* __restrict__ rhs, const T* __restrict__ p_in, T* __restrict__ p_out,
                       float dx2, float omega, const double* __restrict__ check, double tol2,
                       double* __restrict__ resid_out, unsigned long long* __restrict__ counters,
                       uint32_t first_polls) {
    __shared__ Stage<T> st[2];
    __shared__ double red[2][NT / 32];
    __shared__ int ok;
    if (check != nullptr && check[0] <= tol2 * check[1]) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t L = t.num_leaves, G = gridDim.x;
    const T* zero = reinterpret_cast<const T*>(g_zero_leaf);
    int64_t leaf = blockIdx.x;

    // The thread's voxels (see above) and copy plan.
    const int k = lane & 3, q = (lane >> 2) & 3, h = (lane >> 4) & 1;
    const int a0 = 2 * (warp >> 1) + h, a1 = a0 + 4, bq = 4 * (warp & 1) + q;
    const int p0 = (a0 + bq) & 1, p1 = (a1 + bq) & 1;
    const Cell red0 = row_cell(a0, bq, 2 * k + p0), red1 = row_cell(a1, bq, 2 * k + p1);
    const Cell blk0 = row_cell(a0, bq, 2 * k + (p0 ^ 1)), blk1 = row_cell(a1, bq, 2 * k + (p1 ^ 1));
    int ring_nb;
    Cell ring;
    if (warp < 2) {  // x-ring row (h ? 8 : -1, 4 warp + q)
        const int a = h ? 8 : -1, b = 4 * warp + q;
        ring_nb = nbi(h ? 1 : -1, 0, 0);
        ring = row_cell(a, b, 2 * k + ((a + b) & 1));
    } else {  // y-ring row (4 (warp - 2) + q, h ? 8 : -1)
        const int a = 4 * (warp - 2) + q, b = h ? 8 : -1;
        ring_nb = nbi(0, h ? 1 : -1, 0);
        ring = row_cell(a, b, 2 * k + ((a + b) & 1));
    }
    // z-ring (warps 0, 1): row (a, b) has its red voxel at z = 8 if a + b is even, else at z = -1.
    const int zrow = (warp & 1) * 32 + lane, za = zrow >> 3, zb = zrow & 7, zhi = ((za + zb) & 1) == 0;
    const int zring_nb = nbi(0, 0, zhi ? 1 : -1);
    const Cell zring = zring_cell(za, zb, zhi);
    const CopyPlan<T> cp = copy_plan<T>(tid);

    if (tid == 0) {
        ptx::mbar_init(&st[0].bar, NT);
        ptx::mbar_init(&st[1].bar, NT);
        ptx::fence_barrier_init();
        ok = 1;
        if (counters != nullptr && blockIdx.x == 0) atomicAdd(counters, 1ull);
    }
    // Threads 0-53 own source-table entry tid: neighbour q of the staged leaf, p (tid < 27) or
    // rhs. nb_next holds neighbour q of the CTA's next leaf.
    const int q_nb = tid < 27 ? tid : tid - 27;
    const T* q_arr = tid < 27 ? p_in : rhs;
    int nb_next = -1;
    if (tid < 54) {
        const int l = __ldg(t.nbr27 + leaf * 27 + q_nb);
        if (tid < 27) st[0].nb[tid] = l;
        st[0].src[tid] = leaf_src(q_arr, l, zero);
        if (leaf + G < L) nb_next = __ldg(t.nbr27 + (leaf + G) * 27 + q_nb);
    }
    __syncthreads();
    stage_issue(st[0], cp, tid);

    double r2 = 0.0, b2 = 0.0;
    for (uint32_t i = 0;; ++i) {
        Stage<T>& cur = st[i & 1];
        Stage<T>& nxt = st[(i & 1) ^ 1];
        const int64_t next = leaf + G;
        // nxt was released by the previous iteration (its readers passed the barriers below and
        // fenced their generic accesses): publish the next leaf's neighbours and copy sources,
        // fetch the neighbours of the leaf after it, and start the next leaf's copies.
        if (tid < 54) {
            if (tid < 27) nxt.nb[tid] = nb_next;
            nxt.src[tid] = leaf_src(q_arr, nb_next, zero);
            nb_next = next + G < L ? __ldg(t.nbr27 + (next + G) * 27 + q_nb) : -1;
        }
        __syncthreads();
        if (next < L) stage_issue(nxt, cp, tid);
        // One thread waits for the current stage (sleeping between polls); the others wait at
        // the CTA barrier. first_polls bounds this first wait (kMaxPolls unless a test lowers it
        // to make the wait give up); the drain waits below keep kMaxPolls.
        if (tid == 0) {
            const uint32_t parity = (i >> 1) & 1;
            if (!ptx::mbar_wait_bounded_sleep(&cur.bar, parity, first_polls, kSuspendNs)) {
                // The copies did not land in time: flag it, and give them and the next stage's
                // copies a second bounded wait so that no copy is still writing when the CTA's
                // shared memory is released. p_out keeps its old values for the leaves left.
                if (counters != nullptr) atomicExch(counters + 1, 1ull);
                (void)ptx::mbar_wait_bounded_sleep(&cur.bar, parity, kMaxPolls, kSuspendNs);
                if (next < L) (void)ptx::mbar_wait_bounded_sleep(&nxt.bar, ((i + 1) >> 1) & 1, kMaxPolls, kSuspendNs);
                ok = 0;
            }
        }
        __syncthreads();
        if (!ok) return;
        T* v = cur.v;

        if (resid_out != nullptr) {
            const double hh = (double)dx2;
            for (int n = tid; n < 512; n += NT) {
                const int a = n >> 6, b = (n >> 3) & 7, d = n & 7;
                const double lap = (double)pv(v, a + 1, b, d) + (double)pv(v, a - 1, b, d) + (double)pv(v, a, b + 1, d) +
                                   (double)pv(v, a, b - 1, d) + (double)pv(v, a, b, d + 1) + (double)pv(v, a, b, d - 1) -
                                   6.0 * (double)pv(v, a, b, d);
                const double bb = (double)bv(v, a, b, d) * hh;
                r2 += (bb - lap) * (bb - lap);
                b2 += bb * bb;
            }
        }

        // Red (colour 0), then black: leaf origins are multiples of 8, so a voxel's colour is
        // the parity of its local a + b + d.
        relax<96, 8>(v, red0, dx2, omega);
        relax<96, 8>(v, red1, dx2, omega);
        if (cur.nb[ring_nb] >= 0) relax<96, 8>(v, ring, dx2, omega);
        if (warp < 2 && cur.nb[zring_nb] >= 0) relax<48, 4>(v, zring, dx2, omega);
        __syncthreads();
        relax<96, 8>(v, blk0, dx2, omega);
        relax<96, 8>(v, blk1, dx2, omega);
        __syncthreads();
        constexpr int kVec = 16 / sizeof(T);  // values per 16-byte store
        if (tid * kVec < 512) {
            const int o = tid * kVec;
            *reinterpret_cast<uint4*>(p_out + (leaf << 9) + o) =
                *reinterpret_cast<const uint4*>(&v[kOffP + prow(o >> 6, 0) * 8 + (o & 63)]);
        }
        ptx::fence_proxy_async_smem();
        leaf = next;
        if (leaf >= L) break;
    }

    if (resid_out != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            b2 += __shfl_xor_sync(0xffffffffu, b2, o);
        }
        if (lane == 0) red[0][warp] = r2, red[1][warp] = b2;
        __syncthreads();
        if (tid == 0) {
            double sr = 0.0, sb = 0.0;
            for (int w = 0; w < NT / 32; ++w) sr += red[0][w], sb += red[1][w];
            atomicAdd(resid_out, sr);
            atomicAdd(resid_out + 1, sb);
        }
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

namespace {

constexpr int kGridCacheDevices = 64;

// Grid of the persistent kernel on the current device: every SM filled with as many CTAs as
// fit (looked up once per device), but no more CTAs than leaves.
template <typename T>
unsigned stream_grid(const Context& c) {
    static std::mutex mu;
    static int cap[kGridCacheDevices] = {};
    if (c.device < 0 || c.device >= kGridCacheDevices) fail(HNS_ERR_UNSUPPORTED, "device ordinal too large");
    int g;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cap[c.device] == 0) {
            int sms = 0, per_sm = 0;
            HNS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
            HNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbgs_stream_kernel<T>, NT, 0));
            cap[c.device] = std::max(1, sms) * std::max(1, per_sm);
        }
        g = cap[c.device];
    }
    return (unsigned)std::min<int64_t>(g, c.topo.num_leaves);
}

template <typename T>
void launch_stream(const Context& c, const T* rhs, const T* p_in, T* p_out, float dx2, float omega,
                   const double* check, double tol2, double* resid_out) {
    if (c.topo.num_leaves <= 0) return;
    const uint32_t first_polls = c.first_wait_polls < 0 ? kMaxPolls : (uint32_t)c.first_wait_polls;
    rbgs_stream_kernel<T><<<stream_grid<T>(c), NT, 0, c.stream>>>(c.topo.view, rhs, p_in, p_out, dx2, omega, check, tol2,
                                                                 resid_out, c.counters, first_polls);
    HNS_LAUNCHED();
}

}  // namespace

void launch_rbgs_bulk(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                      const double* check, double tol2, double* resid_out) {
    launch_stream<float>(c, div, p_in, p_out, c.dx * c.dx, omega, check, tol2, resid_out);
}

void launch_rbgs_bulk_unit(const Context& c, const float* rhs, const float* e_in, float* e_out, float omega,
                           const double* check, double tol2) {
    if (!aligned16(rhs) || !aligned16(e_in) || !aligned16(e_out)) fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be 16-byte aligned");
    launch_stream<float>(c, rhs, e_in, e_out, 1.0f, omega, check, tol2, nullptr);
}

void launch_rbgs_bulk_half(const Context& c, const void* rhs, const void* e_in, void* e_out, float omega,
                           const double* check, double tol2) {
    const __half* r = static_cast<const __half*>(rhs);
    const __half* ei = static_cast<const __half*>(e_in);
    __half* eo = static_cast<__half*>(e_out);
    if (!aligned16(r) || !aligned16(ei) || !aligned16(eo)) fail(HNS_ERR_INVALID_ARG, "inner-solve arrays must be 16-byte aligned");
    launch_stream<__half>(c, r, ei, eo, 1.0f, omega, check, tol2, nullptr);
}

}  // namespace hns
