// Host side of libhns: errors, device memory, topology tables, the context and the C ABI
// of include/hns.h.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "hns_internal.cuh"

namespace hns {

// ---- errors --------------------------------------------------------------------------------

namespace {
thread_local std::string g_last_error;
}

void fail(hns_status s, const std::string& msg) { throw Error(s, msg); }

void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return;
    const hns_status s = (e == cudaErrorMemoryAllocation) ? HNS_ERR_OUT_OF_MEMORY : HNS_ERR_CUDA;
    throw Error(s, std::string(cudaGetErrorString(e)) + " in " + what + " (" + file + ":" + std::to_string(line) + ")");
}

hns_status record_error(hns_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

void clear_error() { g_last_error.clear(); }

// ---- device memory ---------------------------------------------------------------------------

void DeviceBuffer::alloc(size_t n) {
    reset();
    if (n == 0) return;
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        fail(HNS_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(n) + " bytes failed: " + cudaGetErrorString(e));
    }
    ptr = p;
    bytes = n;
}

void DeviceBuffer::reset() noexcept {
    if (ptr) (void)cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

DeviceGuard::DeviceGuard(int dev) {
    HNS_CUDA(cudaGetDevice(&prev));
    if (prev != dev) HNS_CUDA(cudaSetDevice(dev));
}

DeviceGuard::~DeviceGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && prev >= 0 && cur != prev) (void)cudaSetDevice(prev);
}

// ---- topology ------------------------------------------------------------------------------

namespace {

struct LeafKey {
    int32_t x, y, z;
    bool operator==(const LeafKey& o) const { return x == o.x && y == o.y && z == o.z; }
};

struct LeafKeyHash {
    size_t operator()(const LeafKey& k) const {
        uint64_t h = (uint64_t)(uint32_t)k.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)k.y * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)k.z * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)(h ^ (h >> 29));
    }
};

// Largest dense leaf table accepted (entries of 4 bytes): 2^28 entries = 1 GiB, e.g. a
// bounding box of 5120^3 voxels.
constexpr int64_t kMaxLookupEntries = int64_t(1) << 28;

// NanoVDB leaf order key: 4096^3 root tile (signed x, y, z), upper-node child index,
// lower-node child index (externals/nanovdb/tools/cuda/PointsToGrid.cuh:596-651).
bool nanovdb_less(const int32_t* a, const int32_t* b) {
    for (int d = 0; d < 3; ++d) {
        const int32_t x = a[d] >> 12, y = b[d] >> 12;
        if (x != y) return x < y;
    }
    for (int d = 0; d < 3; ++d) {
        const int32_t x = (a[d] >> 7) & 31, y = (b[d] >> 7) & 31;
        if (x != y) return x < y;
    }
    for (int d = 0; d < 3; ++d) {
        const int32_t x = (a[d] >> 3) & 15, y = (b[d] >> 3) & 15;
        if (x != y) return x < y;
    }
    return false;
}

}  // namespace

bool leaves_in_nanovdb_order(const int32_t* o, int64_t n) {
    for (int64_t i = 1; i < n; ++i)
        if (!nanovdb_less(o + 3 * (i - 1), o + 3 * i)) return false;
    return true;
}

void sort_leaves_nanovdb(int32_t* o, int64_t n) {
    std::vector<int64_t> idx(n);
    for (int64_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return nanovdb_less(o + 3 * a, o + 3 * b); });
    std::vector<int32_t> tmp(o, o + 3 * n);
    for (int64_t i = 0; i < n; ++i) std::memcpy(o + 3 * i, tmp.data() + 3 * idx[i], 3 * sizeof(int32_t));
}

void Topology::build(const int32_t* leaf_origins, int64_t n, cudaStream_t stream) {
    if (n <= 0) fail(HNS_ERR_INVALID_ARG, "topology needs at least one leaf");
    if (n > (int64_t(1) << 31) - 1) fail(HNS_ERR_UNSUPPORTED, "more than 2^31-1 leaves");
    num_leaves = n;
    origins.assign(leaf_origins, leaf_origins + 3 * n);
    std::unordered_map<LeafKey, int32_t, LeafKeyHash> index;
    index.reserve((size_t)n * 2);
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t l = 0; l < n; ++l) {
        const int32_t* o = leaf_origins + 3 * l;
        if ((o[0] & 7) || (o[1] & 7) || (o[2] & 7))
            fail(HNS_ERR_LAYOUT, "leaf " + std::to_string(l) + " origin is not a multiple of 8");
        const LeafKey key{o[0] >> 3, o[1] >> 3, o[2] >> 3};
        if (!index.emplace(key, (int32_t)l).second) fail(HNS_ERR_LAYOUT, "leaf " + std::to_string(l) + " is repeated");
        lo[0] = std::min(lo[0], key.x), lo[1] = std::min(lo[1], key.y), lo[2] = std::min(lo[2], key.z);
        hi[0] = std::max(hi[0], key.x), hi[1] = std::max(hi[1], key.y), hi[2] = std::max(hi[2], key.z);
    }
    nanovdb_order = leaves_in_nanovdb_order(leaf_origins, n);

    const int64_t dims[3] = {int64_t(hi[0]) - lo[0] + 1, int64_t(hi[1]) - lo[1] + 1, int64_t(hi[2]) - lo[2] + 1};
    const int64_t entries = dims[0] * dims[1] * dims[2];
    if (dims[0] > INT32_MAX || dims[1] > INT32_MAX || dims[2] > INT32_MAX || entries > kMaxLookupEntries)
        fail(HNS_ERR_UNSUPPORTED, "leaf bounding box of " + std::to_string(dims[0]) + "x" + std::to_string(dims[1]) + "x" +
                                      std::to_string(dims[2]) + " leaves exceeds the dense leaf table limit of 2^28 entries");
    std::vector<int32_t> lookup((size_t)entries, -1);
    std::vector<int4> org((size_t)n);
    std::vector<int32_t> nbr((size_t)n * 27);
    for (int64_t l = 0; l < n; ++l) {
        const int32_t* o = leaf_origins + 3 * l;
        const int32_t a = o[0] >> 3, b = o[1] >> 3, c = o[2] >> 3;
        org[l] = make_int4(o[0], o[1], o[2], 0);
        lookup[((size_t)(a - lo[0]) * dims[1] + (b - lo[1])) * dims[2] + (c - lo[2])] = (int32_t)l;
    }
    for (int64_t l = 0; l < n; ++l) {
        const int32_t* o = leaf_origins + 3 * l;
        const int32_t a = o[0] >> 3, b = o[1] >> 3, c = o[2] >> 3;
        for (int q = 0; q < 27; ++q) {
            const int64_t x = int64_t(a) + q / 9 - 1, y = int64_t(b) + (q / 3) % 3 - 1, z = int64_t(c) + q % 3 - 1;
            int32_t v = -1;
            if (x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2])
                v = lookup[((size_t)(x - lo[0]) * dims[1] + (y - lo[1])) * dims[2] + (z - lo[2])];
            nbr[(size_t)l * 27 + q] = v;
        }
    }
    d_origin.alloc(sizeof(int4) * (size_t)n);
    d_nbr27.alloc(sizeof(int32_t) * nbr.size());
    d_lookup.alloc(sizeof(int32_t) * lookup.size());
    HNS_CUDA(cudaMemcpyAsync(d_origin.ptr, org.data(), d_origin.bytes, cudaMemcpyHostToDevice, stream));
    HNS_CUDA(cudaMemcpyAsync(d_nbr27.ptr, nbr.data(), d_nbr27.bytes, cudaMemcpyHostToDevice, stream));
    HNS_CUDA(cudaMemcpyAsync(d_lookup.ptr, lookup.data(), d_lookup.bytes, cudaMemcpyHostToDevice, stream));
    HNS_CUDA(cudaStreamSynchronize(stream));  // host vectors go out of scope
    view.num_leaves = n;
    view.origin = d_origin.as<int4>();
    view.nbr27 = d_nbr27.as<int>();
    view.lookup = d_lookup.as<int>();
    view.lo_x = lo[0], view.lo_y = lo[1], view.lo_z = lo[2];
    view.dim_x = (int)dims[0], view.dim_y = (int)dims[1], view.dim_z = (int)dims[2];
}

// ---- context ---------------------------------------------------------------------------------

float* Context::scratch_f32(const std::string& name, size_t count) {
    DeviceBuffer& b = scratch[name];
    if (b.bytes < count * sizeof(float)) b.alloc(count * sizeof(float));
    return b.as<float>();
}

bool Context::stream_capturing() const {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    HNS_CUDA(cudaStreamIsCapturing(stream, &st));
    return st != cudaStreamCaptureStatusNone;
}

void Context::release_spare_graphs() {
    for (auto& g : spare_graphs) {
        if (g.exec) (void)cudaGraphExecDestroy(g.exec);
        if (g.graph) (void)cudaGraphDestroy(g.graph);
    }
    spare_graphs.clear();
}

double* Context::reduce_slots(int count) {
    if (count > kReduceSlots) fail(HNS_ERR_UNSUPPORTED, "more than " + std::to_string(kMaxChecks) + " convergence checks");
    if (!d_reduce.ptr) d_reduce.alloc(sizeof(double) * kReduceSlots);
    return d_reduce.as<double>();
}

std::atomic<unsigned long long> g_kernel_launches{0};
void note_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

int Context::sm_count() const {
    if (sms == 0) HNS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return sms;
}

void Context::ensure_aux() {
    if (aux_stream == nullptr) HNS_CUDA(cudaStreamCreateWithFlags(&aux_stream, cudaStreamNonBlocking));
    if (aux_ready == nullptr) HNS_CUDA(cudaEventCreateWithFlags(&aux_ready, cudaEventDisableTiming));
}

void Context::phase_begin(int phase) {
    if (!profiling) return;
    PhaseEvent e{phase, nullptr, nullptr};
    HNS_CUDA(cudaEventCreate(&e.start));
    HNS_CUDA(cudaEventCreate(&e.stop));
    HNS_CUDA(cudaEventRecord(e.start, stream));
    phase_events.push_back(e);
    open_phases.push_back(phase_events.size() - 1);
}

void Context::phase_end() {
    if (!profiling || open_phases.empty()) return;
    HNS_CUDA(cudaEventRecord(phase_events[open_phases.back()].stop, stream));
    open_phases.pop_back();
}

Context* check_ctx(hns_ctx* ctx) {
    if (!ctx) fail(HNS_ERR_INVALID_ARG, "null context");
    return &ctx->impl;
}

const Context* check_ctx(const hns_ctx* ctx) {
    if (!ctx) fail(HNS_ERR_INVALID_ARG, "null context");
    return &ctx->impl;
}

void rbgs_solve(Context& c, const float* div, float* p, int iterations, float omega, unsigned flags) {
    if (iterations <= 0) {
        if (flags & HNS_SOLVE_ZERO_INIT) HNS_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * c.num_voxels(), c.stream));
        return;
    }
    if (use_split32(c, flags, div, p)) {
        split32_solve(c, div, p, iterations, omega, flags, nullptr);
        return;
    }
    const size_t n = (size_t)c.num_voxels();
    float* tmp = c.scratch_f32("rbgs_pingpong", n);
    // Ping-pong so that the last iteration writes into p.
    float* buf[2];
    const float* src;
    if (flags & HNS_SOLVE_ZERO_INIT) {
        src = nullptr;
        buf[0] = (iterations & 1) ? p : tmp;
        buf[1] = (iterations & 1) ? tmp : p;
    } else if (iterations & 1) {
        HNS_CUDA(cudaMemcpyAsync(tmp, p, sizeof(float) * n, cudaMemcpyDeviceToDevice, c.stream));
        src = tmp;
        buf[0] = p;
        buf[1] = tmp;
    } else {
        src = p;
        buf[0] = tmp;
        buf[1] = p;
    }
    for (int it = 0; it < iterations; ++it) {
        float* dst = buf[it & 1];
        launch_rbgs_iteration(c, div, src, dst, omega, flags);
        src = dst;
    }
}

}  // namespace hns

using namespace hns;

namespace {

void check_ptr(const void* p, const char* what) {
    if (!p) fail(HNS_ERR_INVALID_ARG, std::string("null ") + what);
}

hns_status create_impl(hns_ctx** out, float voxel_size, int device, const std::function<void(Context&)>& build_topology) {
    return guarded([&] {
        check_ptr(out, "output pointer");
        *out = nullptr;
        if (!(voxel_size > 0.f) || !std::isfinite(voxel_size)) fail(HNS_ERR_INVALID_ARG, "voxel size must be positive and finite");
        int count = 0;
        HNS_CUDA(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) fail(HNS_ERR_INVALID_ARG, "device ordinal out of range");
        DeviceGuard g(device);
        auto ctx = std::make_unique<hns_ctx>();
        Context& c = ctx->impl;
        c.device = device;
        c.dx = voxel_size;
        HNS_CUDA(cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking));
        c.stream = c.own_stream;
        try {
            build_topology(c);
            c.d_counters.alloc(sizeof(unsigned long long) * 8);
            c.counters = c.d_counters.as<unsigned long long>();
            HNS_CUDA(cudaMemsetAsync(c.counters, 0, c.d_counters.bytes, c.stream));
            c.reduce_slots(1);
            c.d_solve_log.alloc(sizeof(double) * (2 * Context::kSolveLogCap + 1));
            HNS_CUDA(cudaMemsetAsync(c.d_solve_log.ptr, 0, c.d_solve_log.bytes, c.stream));
        } catch (...) {
            (void)cudaStreamDestroy(c.own_stream);
            c.own_stream = nullptr;
            throw;
        }
        *out = ctx.release();
    });
}

}  // namespace

extern "C" {

HNS_API int hns_abi_version(void) { return HNS_ABI_VERSION; }

HNS_API const char* hns_status_string(hns_status s) {
    switch (s) {
        case HNS_OK: return "ok";
        case HNS_ERR_INVALID_ARG: return "invalid argument";
        case HNS_ERR_CUDA: return "CUDA error";
        case HNS_ERR_OUT_OF_MEMORY: return "out of device memory";
        case HNS_ERR_NOT_FOUND: return "not found";
        case HNS_ERR_LAYOUT: return "invalid leaf layout";
        case HNS_ERR_NOT_CONVERGED: return "not converged";
        case HNS_ERR_UNSUPPORTED: return "unsupported";
        case HNS_ERR_TIMEOUT: return "device wait timed out";
    }
    return "unknown status";
}

HNS_API const char* hns_last_error(void) { return g_last_error.c_str(); }

HNS_API hns_status hns_create(hns_ctx** out, const int32_t* leaf_origins, int64_t num_leaves, float voxel_size, int device) {
    if (!leaf_origins) return record_error(HNS_ERR_INVALID_ARG, "null leaf origins");
    return create_impl(out, voxel_size, device, [&](Context& c) { c.topo.build(leaf_origins, num_leaves, c.stream); });
}

HNS_API hns_status hns_create_from_voxels(hns_ctx** out, const int32_t* ijk, int64_t num_voxels, int padding,
                                          int ijk_on_device, float voxel_size, int device) {
    if (!ijk) return record_error(HNS_ERR_INVALID_ARG, "null voxel coordinates");
    return create_impl(out, voxel_size, device, [&](Context& c) {
        c.topo.build_from_voxels(ijk, num_voxels, ijk_on_device != 0, padding, c.stream);
    });
}

HNS_API hns_status hns_create_from_coords(hns_ctx** out, const int32_t* coords, int64_t num_voxels, float voxel_size,
                                          int device) {
    std::vector<int32_t> origins;
    const hns_status s = guarded([&] {
        check_ptr(out, "output pointer");
        *out = nullptr;
        check_ptr(coords, "coordinates");
        if (num_voxels <= 0 || num_voxels % 512 != 0)
            fail(HNS_ERR_LAYOUT, "voxel count " + std::to_string(num_voxels) + " is not a positive multiple of 512");
        const int64_t L = num_voxels / 512;
        origins.resize((size_t)L * 3);
        for (int64_t l = 0; l < L; ++l) {
            const int32_t* c0 = coords + 3 * (l * 512);
            for (int d = 0; d < 3; ++d) origins[3 * l + d] = c0[d];
            for (int q = 0; q < 512; ++q) {
                const int32_t* c = coords + 3 * (l * 512 + q);
                if (c[0] != c0[0] + ((q >> 6) & 7) || c[1] != c0[1] + ((q >> 3) & 7) || c[2] != c0[2] + (q & 7))
                    fail(HNS_ERR_LAYOUT, "slot " + std::to_string(l * 512 + q) + " is not leaf-dense (x-major 8^3 leaves)");
            }
        }
    });
    if (s != HNS_OK) return s;
    return create_impl(out, voxel_size, device,
                       [&](Context& c) { c.topo.build(origins.data(), (int64_t)origins.size() / 3, c.stream); });
}

HNS_API hns_status hns_destroy(hns_ctx* ctx) {
    if (!ctx) return HNS_OK;
    return guarded([&] {
        Context& c = ctx->impl;
        DeviceGuard g(c.device);
        if (c.stream) (void)cudaStreamSynchronize(c.stream);
        if (c.aux_stream) {
            (void)cudaStreamSynchronize(c.aux_stream);
            (void)cudaStreamDestroy(c.aux_stream);
        }
        if (c.aux_ready) (void)cudaEventDestroy(c.aux_ready);
        if (c.refine_echo_done) (void)cudaEventDestroy(c.refine_echo_done);
        if (c.refine_echo) (void)cudaFreeHost(c.refine_echo);
        c.release_staging();
        c.release_spare_graphs();
        for (auto& e : c.phase_events) {
            (void)cudaEventDestroy(e.start);
            (void)cudaEventDestroy(e.stop);
        }
        c.phase_events.clear();
        if (c.own_stream) (void)cudaStreamDestroy(c.own_stream);
        delete ctx;
    });
}

HNS_API hns_status hns_set_stream(hns_ctx* ctx, void* stream) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    });
}

HNS_API void* hns_get_stream(const hns_ctx* ctx) { return ctx ? (void*)ctx->impl.stream : nullptr; }

HNS_API hns_status hns_synchronize(hns_ctx* ctx) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        DeviceGuard g(c->device);
        HNS_CUDA(cudaStreamSynchronize(c->stream));
    });
}

HNS_API int64_t hns_num_voxels(const hns_ctx* ctx) { return ctx ? ctx->impl.num_voxels() : 0; }
HNS_API int64_t hns_num_leaves(const hns_ctx* ctx) { return ctx ? ctx->impl.topo.num_leaves : 0; }
HNS_API float hns_voxel_size(const hns_ctx* ctx) { return ctx ? ctx->impl.dx : 0.f; }

HNS_API hns_status hns_set_option(hns_ctx* ctx, int option, int value) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (option == HNS_OPT_RBGS_KERNEL) {
            if (value != HNS_RBGS_PLAIN && value != HNS_RBGS_BULK && value != HNS_RBGS_SPLIT)
                fail(HNS_ERR_INVALID_ARG, "unknown red-black kernel");
            c->rbgs_kernel = value;
        } else if (option == HNS_OPT_INNER_LAYOUT) {
            if (value != HNS_INNER_ROWS && value != HNS_INNER_PACKED && value != HNS_INNER_SPLIT)
                fail(HNS_ERR_INVALID_ARG, "unknown inner layout");
            c->inner_layout = value;
        } else if (option == HNS_OPT_SPLIT_SOLVE) {
            if (value != HNS_SPLIT_PER_COLOUR && value != HNS_SPLIT_PERSISTENT)
                fail(HNS_ERR_INVALID_ARG, "unknown inner-solve launch form");
            c->split_solve = value;
        } else if (option == HNS_OPT_COARSE_SOLVE) {
            if (value != HNS_COARSE_LAUNCHES && value != HNS_COARSE_CLUSTER)
                fail(HNS_ERR_INVALID_ARG, "unknown coarse-level solve");
            c->coarse_solve = value;
        } else if (option == HNS_OPT_L2_PERSIST) {
            if (value != 0 && value != 1) fail(HNS_ERR_INVALID_ARG, "HNS_OPT_L2_PERSIST takes 0 or 1");
            c->l2_persist = value;
        } else if (option == HNS_OPT_WAIT_POLLS) {
            if (value < -1) fail(HNS_ERR_INVALID_ARG, "the wait limit must be -1 (default) or >= 0");
            c->first_wait_polls = value;
        } else {
            fail(HNS_ERR_INVALID_ARG, "unknown option");
        }
    });
}

HNS_API hns_status hns_device_status(hns_ctx* ctx) {
    unsigned long long flag = 0;
    const hns_status s = guarded([&] {
        Context* c = check_ctx(ctx);
        DeviceGuard g(c->device);
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        HNS_CUDA(cudaMemcpy(&flag, c->counters + 1, sizeof(flag), cudaMemcpyDeviceToHost));
        if (flag) {
            HNS_CUDA(cudaMemsetAsync(c->counters + 1, 0, sizeof(flag), c->stream));
            HNS_CUDA(cudaStreamSynchronize(c->stream));
        }
    });
    if (s != HNS_OK) return s;
    return flag ? record_error(HNS_ERR_TIMEOUT, "a device-side wait gave up (a bulk copy or a neighbour's sweep did not complete)") : HNS_OK;
}

HNS_API hns_status hns_profile_enable(hns_ctx* ctx, int enable) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        c->profiling = enable != 0;
    });
}

HNS_API hns_status hns_profile_read(hns_ctx* ctx, hns_profile_data* out) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(out, "output");
        DeviceGuard g(c->device);
        std::memset(out, 0, sizeof(*out));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        for (auto& e : c->phase_events) {
            float ms = 0.f;
            HNS_CUDA(cudaEventElapsedTime(&ms, e.start, e.stop));
            if (e.phase >= 0 && e.phase < HNS_NUM_PHASES) {
                out->phase_ms[e.phase] += ms;
                out->phase_count[e.phase] += 1;
            }
            (void)cudaEventDestroy(e.start);
            (void)cudaEventDestroy(e.stop);
        }
        c->phase_events.clear();
        HNS_CUDA(cudaMemcpy(&out->solver_launches, c->counters, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        HNS_CUDA(cudaMemsetAsync(c->counters, 0, sizeof(unsigned long long), c->stream));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        out->kernel_launches = ::hns::g_kernel_launches.exchange(0, std::memory_order_relaxed);
    });
}

HNS_API hns_status hns_leaf_origins(const hns_ctx* ctx, int32_t* out) {
    return guarded([&] {
        const Context* c = check_ctx(ctx);
        check_ptr(out, "output");
        std::memcpy(out, c->topo.origins.data(), c->topo.origins.size() * sizeof(int32_t));
    });
}

HNS_API hns_status hns_index_offsets(hns_ctx* ctx, const int32_t* ijk, int64_t n, uint64_t* out) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (n < 0) fail(HNS_ERR_INVALID_ARG, "negative count");
        if (n == 0) return;
        check_ptr(ijk, "coordinates");
        check_ptr(out, "output");
        DeviceGuard g(c->device);
        DeviceBuffer d_ijk(sizeof(int32_t) * 3 * (size_t)n), d_out(sizeof(uint64_t) * (size_t)n);
        HNS_CUDA(cudaMemcpyAsync(d_ijk.ptr, ijk, d_ijk.bytes, cudaMemcpyHostToDevice, c->stream));
        launch_index_offsets(*c, d_ijk.as<int32_t>(), n, d_out.as<uint64_t>());
        HNS_CUDA(cudaMemcpyAsync(out, d_out.ptr, d_out.bytes, cudaMemcpyDeviceToHost, c->stream));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
    });
}

HNS_API hns_status hns_sort_leaves_nanovdb(int32_t* leaf_origins, int64_t n) {
    return guarded([&] {
        if (n < 0) fail(HNS_ERR_INVALID_ARG, "negative count");
        if (n > 0) check_ptr(leaf_origins, "leaf origins");
        sort_leaves_nanovdb(leaf_origins, n);
    });
}

HNS_API hns_status hns_is_nanovdb_order(const hns_ctx* ctx, int* out) {
    return guarded([&] {
        const Context* c = check_ctx(ctx);
        check_ptr(out, "output");
        *out = c->topo.nanovdb_order ? 1 : 0;
    });
}

// ---- operators -----------------------------------------------------------------------------

HNS_API hns_status hns_advect_vec3(hns_ctx* ctx, const float* vel, float* out, float dt) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        check_ptr(out, "output");
        if (vel == out) fail(HNS_ERR_INVALID_ARG, "advection cannot run in place");
        DeviceGuard g(c->device);
        FieldSet none{};
        launch_advect_fused(*c, vel, out, none, dt);
    });
}

HNS_API hns_status hns_advect_scalar(hns_ctx* ctx, const float* vel, const float* in, float* out, float dt) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        check_ptr(in, "input");
        check_ptr(out, "output");
        if (in == out) fail(HNS_ERR_INVALID_ARG, "advection cannot run in place");
        DeviceGuard g(c->device);
        FieldSet f{};
        f.count = 1;
        f.in[0] = in;
        f.out[0] = out;
        launch_advect_fused(*c, vel, nullptr, f, dt);
    });
}

HNS_API hns_status hns_advect_scalars(hns_ctx* ctx, const float* vel, const float* const* in, float* const* out,
                                      int nfields, float dt) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        if (nfields < 0) fail(HNS_ERR_INVALID_ARG, "negative field count");
        if (nfields == 0) return;
        check_ptr(in, "input array");
        check_ptr(out, "output array");
        DeviceGuard g(c->device);
        for (int base = 0; base < nfields; base += kMaxAdvectFields) {
            FieldSet f{};
            f.count = std::min(kMaxAdvectFields, nfields - base);
            for (int q = 0; q < f.count; ++q) {
                check_ptr(in[base + q], "input field");
                check_ptr(out[base + q], "output field");
                f.in[q] = in[base + q];
                f.out[q] = out[base + q];
            }
            for (int q = 0; q < f.count; ++q)
                for (int r = 0; r < nfields; ++r)
                    if (f.out[q] == in[r]) fail(HNS_ERR_INVALID_ARG, "advection outputs cannot alias inputs");
            launch_advect_scalars(*c, vel, f, dt);
        }
    });
}

HNS_API hns_status hns_divergence(hns_ctx* ctx, const float* vel, float* div) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        check_ptr(div, "output");
        DeviceGuard g(c->device);
        launch_divergence(*c, vel, div);
    });
}

HNS_API hns_status hns_rbgs(hns_ctx* ctx, const float* div, float* p, int iterations, float omega, unsigned flags) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(div, "divergence");
        check_ptr(p, "pressure");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        DeviceGuard g(c->device);
        rbgs_solve(*c, div, p, iterations, omega, flags);
    });
}

HNS_API hns_status hns_subtract_gradient(hns_ctx* ctx, const float* vel, const float* p, float* out) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        check_ptr(p, "pressure");
        check_ptr(out, "output");
        DeviceGuard g(c->device);
        launch_subtract_gradient(*c, vel, p, out);
    });
}

HNS_API hns_status hns_vorticity_confinement(hns_ctx* ctx, const float* vel, float* out, float dt, float scale,
                                             float factor_scale) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        check_ptr(out, "output");
        if (vel == out) fail(HNS_ERR_INVALID_ARG, "vorticity confinement cannot run in place");
        if (!std::isfinite(factor_scale) || std::fabs(factor_scale) > 1e6f) fail(HNS_ERR_INVALID_ARG, "factor_scale out of range");
        DeviceGuard g(c->device);
        launch_vorticity(*c, vel, out, dt, scale, factor_scale);
    });
}

HNS_API hns_status hns_project(hns_ctx* ctx, float* vel, int iterations, float omega, unsigned flags, hns_solve_info* info) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        check_ptr(vel, "velocity");
        if (((uintptr_t)vel & 3u) != 0) fail(HNS_ERR_INVALID_ARG, "velocity must be 4-byte aligned");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        DeviceGuard g(c->device);
        const size_t n = (size_t)c->num_voxels();
        if (!(omega > 0.f)) omega = (float)(2.0f / (1.0f + std::sin(3.14159 * (double)c->dx)));
        float* div = c->scratch_f32("project_div", n);
        float* p = c->scratch_f32("project_p", n);
        launch_divergence(*c, vel, div);
        if (flags & HNS_SOLVE_NEUMANN) remove_divergence_mean(*c, div);  // the singular system's compatibility
        double* acc = nullptr;
        if (info) {
            acc = c->reduce_slots(4);
            HNS_CUDA(cudaMemsetAsync(acc, 0, 4 * sizeof(double), c->stream));
            HNS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(float), c->stream));
            launch_residual(*c, div, p, acc, flags);
        }
        rbgs_solve(*c, div, p, iterations, omega, flags | HNS_SOLVE_ZERO_INIT);
        if (info) launch_residual(*c, div, p, acc + 2, flags);
        launch_subtract_gradient(*c, vel, p, vel, nullptr, flags);  // pointwise in vel: safe in place
        if (info) {
            double h[4];
            HNS_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
            HNS_CUDA(cudaStreamSynchronize(c->stream));
            info->iterations = iterations;
            info->initial_residual = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
            info->residual = h[3] > 0 ? std::sqrt(h[2] / h[3]) : 0.0;
        }
    });
}

}  // extern "C"
