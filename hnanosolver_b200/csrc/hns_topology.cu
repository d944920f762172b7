// Topology built on the device from a list of active voxels: the replacement for the
// reference's domain set-up -- the velocity grid's topology dilated by `padding` voxels with
// 26-neighbour (face, edge and vertex) dilation (src/SOP/HNanoSolver/SOP_HNanoSolver.cpp:280-285)
// and the ValueOnIndex grid built from the voxel list with voxelsToGrid
// (src/Cuda/HNanoSolver.cu:498-504). The solver's grids are leaf-dense, so the build produces
// the set of leaves that the dilated voxels touch, in NanoVDB leaf order, and the leaf tables.
//
//   1. Per voxel: its leaf's 63-bit key, which both identifies the leaf and sorts in NanoVDB
//      order (root tile, then upper-node child, then lower-node child; PointsToGrid orders
//      leaves this way), and a 27-bit mask of the neighbour leaves its dilation box reaches
//      (per axis: -1 when z & 7 < padding, +1 when (z & 7) + padding >= 8).
//   2. Radix sort of (key, mask) pairs, reduce-by-key with OR: the active leaves and the
//      union of their reach masks.
//   3. Each active leaf emits the keys of the leaves its mask names; sort and unique: the
//      dilated leaf set, already in NanoVDB order.
//   4. Leaf origins from the keys, the dense leaf table and the 27-neighbour table, on the
//      device; only the origins go back to the host (the context keeps a host copy).
// Library primitives (CUB radix sort, scan, reduce-by-key, unique) do the sorting; this is the
// set-up before the step, not the step's hot path.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "hns_internal.cuh"

namespace hns {
namespace {

constexpr int kTopoThreads = 256;
// |coordinate| bound: the key holds a 12-bit biased root tile index per axis (coordinate >> 12).
constexpr int32_t kCoordLimit = (1 << 23) - 64;
constexpr int kMaxPadding = 8;

unsigned grid_for(int64_t n) { return (unsigned)((n + kTopoThreads - 1) / kTopoThreads); }

__device__ __forceinline__ uint64_t leaf_key(int i, int j, int k) {
    const uint64_t rx = (uint64_t)((i >> 12) + 2048), ry = (uint64_t)((j >> 12) + 2048), rz = (uint64_t)((k >> 12) + 2048);
    return (rx << 51) | (ry << 39) | (rz << 27) | ((uint64_t)((i >> 7) & 31) << 22) | ((uint64_t)((j >> 7) & 31) << 17) |
           ((uint64_t)((k >> 7) & 31) << 12) | ((uint64_t)((i >> 3) & 15) << 8) | ((uint64_t)((j >> 3) & 15) << 4) |
           (uint64_t)((k >> 3) & 15);
}

__device__ __forceinline__ int3 key_origin(uint64_t key) {
    const int rx = (int)((key >> 51) & 4095) - 2048, ry = (int)((key >> 39) & 4095) - 2048,
              rz = (int)((key >> 27) & 4095) - 2048;
    const int ux = (int)((key >> 22) & 31), uy = (int)((key >> 17) & 31), uz = (int)((key >> 12) & 31);
    const int lx = (int)((key >> 8) & 15), ly = (int)((key >> 4) & 15), lz = (int)(key & 15);
    return make_int3(rx * 4096 + ux * 128 + lx * 8, ry * 4096 + uy * 128 + ly * 8, rz * 4096 + uz * 128 + lz * 8);
}

// Step 1. bad[0] is set when a coordinate is out of range.
__global__ void voxel_key_kernel(const int32_t* __restrict__ ijk, int64_t n, int padding, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ masks, int* __restrict__ bad) {
    const int64_t q = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (q >= n) return;
    const int i = ijk[3 * q], j = ijk[3 * q + 1], k = ijk[3 * q + 2];
    if (i <= -kCoordLimit || i >= kCoordLimit || j <= -kCoordLimit || j >= kCoordLimit || k <= -kCoordLimit ||
        k >= kCoordLimit) {
        atomicExch(bad, 1);
        keys[q] = 0;
        masks[q] = 0;
        return;
    }
    keys[q] = leaf_key(i, j, k);
    // Neighbour offsets the box [x - padding, x + padding] reaches, per axis (bit 0: -1, 1: 0, 2: +1).
    auto reach = [padding](int c) { return 2u | ((c & 7) < padding ? 1u : 0u) | ((c & 7) + padding >= 8 ? 4u : 0u); };
    const uint32_t rx = reach(i), ry = reach(j), rz = reach(k);
    uint32_t m = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (((rx >> a) & 1u) && ((ry >> b) & 1u) && ((rz >> c) & 1u)) m |= 1u << (a * 9 + b * 3 + c);
    masks[q] = m;
}

struct BitOr {
    __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a | b; }
};

__global__ void count_kernel(const uint32_t* __restrict__ masks, const int* __restrict__ num, int* __restrict__ counts) {
    const int64_t l = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (l < *num) counts[l] = __popc(masks[l]);
}

// Step 3: the keys of the leaves each active leaf's mask names.
__global__ void expand_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ masks,
                              const int* __restrict__ offsets, const int* __restrict__ num, uint64_t* __restrict__ out) {
    const int64_t l = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (l >= *num) return;
    const int3 o = key_origin(keys[l]);
    uint32_t m = masks[l];
    int w = offsets[l];
    while (m) {
        const int q = __ffs(m) - 1;
        m &= m - 1;
        out[w++] = leaf_key(o.x + 8 * (q / 9 - 1), o.y + 8 * ((q / 3) % 3 - 1), o.z + 8 * (q % 3 - 1));
    }
}

__global__ void origin_kernel(const uint64_t* __restrict__ keys, int64_t n, int4* __restrict__ org) {
    const int64_t l = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (l >= n) return;
    const int3 o = key_origin(keys[l]);
    org[l] = make_int4(o.x, o.y, o.z, 0);
}

__global__ void lookup_fill_kernel(const int4* __restrict__ org, int64_t n, TopoView t, int* __restrict__ lookup) {
    const int64_t l = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (l >= n) return;
    const int4 o = org[l];
    const int64_t a = (o.x >> 3) - t.lo_x, b = (o.y >> 3) - t.lo_y, c = (o.z >> 3) - t.lo_z;
    lookup[(a * t.dim_y + b) * t.dim_z + c] = (int)l;
}

__global__ void nbr27_kernel(const int4* __restrict__ org, int64_t n, TopoView t, int* __restrict__ nbr) {
    const int64_t l = (int64_t)blockIdx.x * kTopoThreads + threadIdx.x;
    if (l >= n) return;
    const int4 o = org[l];
    for (int q = 0; q < 27; ++q) {
        const int a = (o.x >> 3) + q / 9 - 1 - t.lo_x, b = (o.y >> 3) + (q / 3) % 3 - 1 - t.lo_y,
                  c = (o.z >> 3) + q % 3 - 1 - t.lo_z;
        int v = -1;
        if ((unsigned)a < (unsigned)t.dim_x && (unsigned)b < (unsigned)t.dim_y && (unsigned)c < (unsigned)t.dim_z)
            v = t.lookup[((int64_t)a * t.dim_y + b) * t.dim_z + c];
        nbr[l * 27 + q] = v;
    }
}

// CUB temporary storage, grown on demand.
struct Temp {
    DeviceBuffer buf;
    void* get(size_t bytes) {
        if (buf.bytes < bytes) buf.alloc(std::max<size_t>(bytes, 256));
        return buf.ptr;
    }
};

}  // namespace

// Largest dense leaf table accepted, as in the host build.
constexpr int64_t kMaxLookupEntriesDevice = int64_t(1) << 28;

void Topology::build_from_voxels(const int32_t* ijk, int64_t n, bool ijk_on_device, int padding, cudaStream_t s) {
    if (n <= 0) fail(HNS_ERR_INVALID_ARG, "no active voxels");
    if (padding < 0 || padding > kMaxPadding) fail(HNS_ERR_INVALID_ARG, "padding must be in [0, 8] voxels");
    if (n > (int64_t(1) << 31) - 1) fail(HNS_ERR_UNSUPPORTED, "more than 2^31-1 active voxels");
    DeviceBuffer d_ijk;
    const int32_t* dv = ijk;
    if (!ijk_on_device) {
        d_ijk.alloc(sizeof(int32_t) * 3 * (size_t)n);
        HNS_CUDA(cudaMemcpyAsync(d_ijk.ptr, ijk, sizeof(int32_t) * 3 * (size_t)n, cudaMemcpyHostToDevice, s));
        dv = d_ijk.as<int32_t>();
    }
    DeviceBuffer keys(sizeof(uint64_t) * n), masks(sizeof(uint32_t) * n), keys2(sizeof(uint64_t) * n),
        masks2(sizeof(uint32_t) * n), small(sizeof(int) * 4);
    int* d_small = small.as<int>();  // [0] bad coordinate, [1] active leaves, [2] candidate count, [3] leaves
    HNS_CUDA(cudaMemsetAsync(d_small, 0, small.bytes, s));
    Temp tmp;
    voxel_key_kernel<<<grid_for(n), kTopoThreads, 0, s>>>(dv, n, padding, keys.as<uint64_t>(), masks.as<uint32_t>(), d_small);
    HNS_LAUNCHED();
    size_t tb = 0;
    HNS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(), masks.as<uint32_t>(),
                                             masks2.as<uint32_t>(), (int)n, 0, 63, s));
    HNS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                             masks.as<uint32_t>(), masks2.as<uint32_t>(), (int)n, 0, 63, s));
    // Active leaves (unique keys) with the OR of their voxels' masks, back into keys / masks.
    HNS_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, tb, keys2.as<uint64_t>(), keys.as<uint64_t>(), masks2.as<uint32_t>(),
                                            masks.as<uint32_t>(), d_small + 1, BitOr(), (int)n, s));
    HNS_CUDA(cub::DeviceReduce::ReduceByKey(tmp.get(tb), tb, keys2.as<uint64_t>(), keys.as<uint64_t>(),
                                            masks2.as<uint32_t>(), masks.as<uint32_t>(), d_small + 1, BitOr(), (int)n, s));
    int h_small[4];
    HNS_CUDA(cudaMemcpyAsync(h_small, d_small, sizeof(h_small), cudaMemcpyDeviceToHost, s));
    HNS_CUDA(cudaStreamSynchronize(s));
    if (h_small[0]) fail(HNS_ERR_INVALID_ARG, "a voxel coordinate is outside +-(2^23 - 64)");
    const int active = h_small[1];
    // Candidates: every leaf an active leaf's mask names (at most 27 per active leaf).
    DeviceBuffer counts(sizeof(int) * ((size_t)active + 1)), offsets(sizeof(int) * ((size_t)active + 1));
    count_kernel<<<grid_for(active), kTopoThreads, 0, s>>>(masks.as<uint32_t>(), d_small + 1, counts.as<int>());
    HNS_LAUNCHED();
    HNS_CUDA(cudaMemsetAsync(counts.as<int>() + active, 0, sizeof(int), s));
    HNS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts.as<int>(), offsets.as<int>(), active + 1, s));
    HNS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, counts.as<int>(), offsets.as<int>(), active + 1, s));
    int total = 0;
    HNS_CUDA(cudaMemcpyAsync(&total, offsets.as<int>() + active, sizeof(int), cudaMemcpyDeviceToHost, s));
    HNS_CUDA(cudaStreamSynchronize(s));
    DeviceBuffer cand(sizeof(uint64_t) * (size_t)total), cand2(sizeof(uint64_t) * (size_t)total);
    expand_kernel<<<grid_for(active), kTopoThreads, 0, s>>>(keys.as<uint64_t>(), masks.as<uint32_t>(), offsets.as<int>(),
                                                            d_small + 1, cand.as<uint64_t>());
    HNS_LAUNCHED();
    HNS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, cand.as<uint64_t>(), cand2.as<uint64_t>(), total, 0, 63, s));
    HNS_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(tb), tb, cand.as<uint64_t>(), cand2.as<uint64_t>(), total, 0, 63, s));
    HNS_CUDA(cub::DeviceSelect::Unique(nullptr, tb, cand2.as<uint64_t>(), cand.as<uint64_t>(), d_small + 3, total, s));
    HNS_CUDA(cub::DeviceSelect::Unique(tmp.get(tb), tb, cand2.as<uint64_t>(), cand.as<uint64_t>(), d_small + 3, total, s));
    int L = 0;
    HNS_CUDA(cudaMemcpyAsync(&L, d_small + 3, sizeof(int), cudaMemcpyDeviceToHost, s));
    HNS_CUDA(cudaStreamSynchronize(s));

    num_leaves = L;
    d_origin.alloc(sizeof(int4) * (size_t)L);
    origin_kernel<<<grid_for(L), kTopoThreads, 0, s>>>(cand.as<uint64_t>(), L, d_origin.as<int4>());
    HNS_LAUNCHED();
    std::vector<int4> org((size_t)L);
    HNS_CUDA(cudaMemcpyAsync(org.data(), d_origin.ptr, d_origin.bytes, cudaMemcpyDeviceToHost, s));
    HNS_CUDA(cudaStreamSynchronize(s));
    origins.resize((size_t)L * 3);
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t l = 0; l < L; ++l) {
        const int32_t v[3] = {org[l].x, org[l].y, org[l].z};
        for (int d = 0; d < 3; ++d) {
            origins[3 * l + d] = v[d];
            lo[d] = std::min(lo[d], v[d] >> 3);
            hi[d] = std::max(hi[d], v[d] >> 3);
        }
    }
    nanovdb_order = true;
    const int64_t dims[3] = {int64_t(hi[0]) - lo[0] + 1, int64_t(hi[1]) - lo[1] + 1, int64_t(hi[2]) - lo[2] + 1};
    const int64_t entries = dims[0] * dims[1] * dims[2];
    if (entries > kMaxLookupEntriesDevice)
        fail(HNS_ERR_UNSUPPORTED, "leaf bounding box exceeds the dense leaf table limit of 2^28 entries");
    d_lookup.alloc(sizeof(int32_t) * (size_t)entries);
    d_nbr27.alloc(sizeof(int32_t) * 27 * (size_t)L);
    HNS_CUDA(cudaMemsetAsync(d_lookup.ptr, 0xFF, d_lookup.bytes, s));  // -1: no leaf
    view.num_leaves = L;
    view.origin = d_origin.as<int4>();
    view.nbr27 = d_nbr27.as<int>();
    view.lookup = d_lookup.as<int>();
    view.lo_x = lo[0], view.lo_y = lo[1], view.lo_z = lo[2];
    view.dim_x = (int)dims[0], view.dim_y = (int)dims[1], view.dim_z = (int)dims[2];
    lookup_fill_kernel<<<grid_for(L), kTopoThreads, 0, s>>>(d_origin.as<int4>(), L, view, d_lookup.as<int>());
    HNS_LAUNCHED();
    nbr27_kernel<<<grid_for(L), kTopoThreads, 0, s>>>(d_origin.as<int4>(), L, view, d_nbr27.as<int>());
    HNS_LAUNCHED();
    HNS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hns
