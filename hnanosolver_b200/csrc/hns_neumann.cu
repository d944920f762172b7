// Zero-gradient (Neumann) walls, the configurations' boundary condition (HNS_SOLVE_NEUMANN):
// the pressure outside the domain equals that of the voxel inside. The reference reads p = 0
// outside (Dirichlet-0, src/Cuda/Kernel.cu:459-489). With zero-gradient walls the Poisson
// operator is singular, one constant per face-connected component of leaves, and the system is
// solvable only when the right-hand side sums to zero over each component: this file removes the
// divergence's mean per component, the sums in FP64. The relaxation, residual and gradient of
// the Neumann form are in hns_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "hns_internal.cuh"

namespace hns {
namespace {

// Per leaf (one CTA of 256 threads, two values each): the FP64 sum of its 512 values into the
// sum of its component.
__global__ void __launch_bounds__(256) component_sum_kernel(const float* __restrict__ div, const int* __restrict__ comp,
                                                            double* __restrict__ sums) {
    __shared__ double red[8];
    const int64_t leaf = blockIdx.x;
    const float* d = div + (leaf << 9);
    double v = (double)__ldg(d + threadIdx.x) + (double)__ldg(d + threadIdx.x + 256);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        atomicAdd(sums + __ldg(comp + leaf), t);
    }
}

// div -= mean of its component (the mean in FP64, subtracted in FP32).
__global__ void __launch_bounds__(256) remove_mean_kernel(float* __restrict__ div, const int* __restrict__ comp,
                                                          const double* __restrict__ sums,
                                                          const double* __restrict__ counts) {
    const int64_t leaf = blockIdx.x;
    const int c = __ldg(comp + leaf);
    const float m = (float)(sums[c] / counts[c]);
    float* d = div + (leaf << 9);
    d[threadIdx.x] = d[threadIdx.x] - m;
    d[threadIdx.x + 256] = d[threadIdx.x + 256] - m;
}

struct Key {
    int32_t x, y, z;
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        return (size_t)((uint64_t)(uint32_t)k.x * 0x9E3779B97F4A7C15ull ^ (uint64_t)(uint32_t)k.y * 0xC2B2AE3D27D4EB4Full ^
                        (uint64_t)(uint32_t)k.z * 0x165667B19E3779F9ull);
    }
};

}  // namespace

// The largest number of face steps, over leaves, from a leaf to the nearest leaf with a missing
// face neighbour (0 when every leaf has one): how many leaves deep the domain is. Computed on the
// host once per context by a breadth-first pass from those boundary leaves.
int max_leaf_depth(Context& c) {
    if (c.leaf_depth >= 0) return c.leaf_depth;
    const int64_t L = c.topo.num_leaves;
    const int32_t* o = c.topo.origins.data();
    std::unordered_map<Key, int32_t, KeyHash> index;
    index.reserve((size_t)L * 2);
    for (int64_t l = 0; l < L; ++l) index.emplace(Key{o[3 * l] >> 3, o[3 * l + 1] >> 3, o[3 * l + 2] >> 3}, (int32_t)l);
    auto neighbours = [&](int32_t l, int32_t out[6]) {
        const Key k{o[3 * l] >> 3, o[3 * l + 1] >> 3, o[3 * l + 2] >> 3};
        const Key nbrs[6] = {{k.x + 1, k.y, k.z}, {k.x - 1, k.y, k.z}, {k.x, k.y + 1, k.z},
                             {k.x, k.y - 1, k.z}, {k.x, k.y, k.z + 1}, {k.x, k.y, k.z - 1}};
        for (int q = 0; q < 6; ++q) {
            const auto it = index.find(nbrs[q]);
            out[q] = it == index.end() ? -1 : it->second;
        }
    };
    std::vector<int32_t> depth((size_t)L, -1), queue;
    queue.reserve((size_t)L);
    for (int64_t l = 0; l < L; ++l) {
        int32_t n[6];
        neighbours((int32_t)l, n);
        if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[3] < 0 || n[4] < 0 || n[5] < 0) {
            depth[(size_t)l] = 0;
            queue.push_back((int32_t)l);
        }
    }
    int deepest = 0;
    for (size_t h = 0; h < queue.size(); ++h) {
        const int32_t l = queue[h];
        int32_t n[6];
        neighbours(l, n);
        for (int32_t m : n)
            if (m >= 0 && depth[(size_t)m] < 0) {
                depth[(size_t)m] = depth[(size_t)l] + 1;
                deepest = std::max(deepest, depth[(size_t)m]);
                queue.push_back(m);
            }
    }
    c.leaf_depth = deepest;
    return deepest;
}

// Face-connected components of the context's leaves, labelled on the host once per context
// (breadth-first over face neighbours) and kept on the device with their voxel counts.
void ensure_components(Context& c) {
    if (c.num_components > 0) return;
    const int64_t L = c.topo.num_leaves;
    const int32_t* o = c.topo.origins.data();
    std::unordered_map<Key, int32_t, KeyHash> index;
    index.reserve((size_t)L * 2);
    for (int64_t l = 0; l < L; ++l) index.emplace(Key{o[3 * l] >> 3, o[3 * l + 1] >> 3, o[3 * l + 2] >> 3}, (int32_t)l);
    std::vector<int32_t> comp((size_t)L, -1), queue;
    std::vector<double> counts;
    queue.reserve((size_t)L);
    int32_t nc = 0;
    for (int64_t l0 = 0; l0 < L; ++l0) {
        if (comp[(size_t)l0] >= 0) continue;
        queue.clear();
        queue.push_back((int32_t)l0);
        comp[(size_t)l0] = nc;
        for (size_t h = 0; h < queue.size(); ++h) {
            const int32_t l = queue[h];
            const Key k{o[3 * l] >> 3, o[3 * l + 1] >> 3, o[3 * l + 2] >> 3};
            const Key nbrs[6] = {{k.x + 1, k.y, k.z}, {k.x - 1, k.y, k.z}, {k.x, k.y + 1, k.z},
                                 {k.x, k.y - 1, k.z}, {k.x, k.y, k.z + 1}, {k.x, k.y, k.z - 1}};
            for (const Key& nk : nbrs) {
                const auto it = index.find(nk);
                if (it != index.end() && comp[(size_t)it->second] < 0) {
                    comp[(size_t)it->second] = nc;
                    queue.push_back(it->second);
                }
            }
        }
        counts.push_back(512.0 * (double)queue.size());
        ++nc;
    }
    c.d_components.alloc(sizeof(int32_t) * (size_t)L);
    c.d_component_counts.alloc(sizeof(double) * (size_t)nc);
    c.d_component_sums.alloc(sizeof(double) * (size_t)nc);
    HNS_CUDA(cudaMemcpyAsync(c.d_components.ptr, comp.data(), c.d_components.bytes, cudaMemcpyHostToDevice, c.stream));
    HNS_CUDA(cudaMemcpyAsync(c.d_component_counts.ptr, counts.data(), c.d_component_counts.bytes, cudaMemcpyHostToDevice,
                             c.stream));
    HNS_CUDA(cudaStreamSynchronize(c.stream));  // the host vectors go out of scope
    c.num_components = nc;
}

void remove_divergence_mean(Context& c, float* div) {
    const int64_t L = c.topo.num_leaves;
    if (L == 0) return;
    ensure_components(c);
    HNS_CUDA(cudaMemsetAsync(c.d_component_sums.ptr, 0, c.d_component_sums.bytes, c.stream));
    component_sum_kernel<<<(unsigned)L, 256, 0, c.stream>>>(div, c.d_components.as<int>(), c.d_component_sums.as<double>());
    HNS_LAUNCHED();
    remove_mean_kernel<<<(unsigned)L, 256, 0, c.stream>>>(div, c.d_components.as<int>(), c.d_component_sums.as<double>(),
                                                          c.d_component_counts.as<double>());
    HNS_LAUNCHED();
}

}  // namespace hns
