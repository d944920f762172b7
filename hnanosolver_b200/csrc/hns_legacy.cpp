// The reference's C++ entry points (include/hns_legacy.hpp) over the C ABI of hns.h.
#include "hns_legacy.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

void ok(hns_status s, const char* where) {
    if (s != HNS_OK) throw std::runtime_error(std::string(where) + ": " + hns_status_string(s) + ": " + hns_last_error());
}

bool is_source(const std::string& n) { return n.rfind("src_", 0) == 0; }

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) throw std::runtime_error("no CUDA device");
    return d;
}

// Leaf origins of leaf-dense coordinates (HNS_ERR_LAYOUT otherwise).
std::vector<int32_t> leaves_of(const HNS::GridIndexedData& data) {
    const size_t n = data.size();
    if (n == 0 || n % 512 != 0 || !data.pCoords())
        throw std::runtime_error("index grid: " + std::to_string(n) + " voxels is not a positive multiple of 512");
    const HNS::Coord* c = data.pCoords();
    std::vector<int32_t> o(n / 512 * 3);
    for (size_t l = 0; l < n / 512; ++l) {
        const HNS::Coord& c0 = c[l * 512];
        o[3 * l] = c0.x, o[3 * l + 1] = c0.y, o[3 * l + 2] = c0.z;
        for (int q = 0; q < 512; ++q) {
            const HNS::Coord& v = c[l * 512 + q];
            if (v.x != c0.x + ((q >> 6) & 7) || v.y != c0.y + ((q >> 3) & 7) || v.z != c0.z + (q & 7))
                throw std::runtime_error("index grid: slot " + std::to_string(l * 512 + q) + " is not leaf-dense");
        }
    }
    return o;
}

std::string velocity_block(const HNS::GridIndexedData& data) {
    const auto names = data.getBlocksOfType<HNS::Vec3f>();
    if (names.empty()) return std::string();
    for (const auto& n : names)
        if (n == "velocity") return n;
    return names[0];
}

std::string single_velocity_block(const HNS::GridIndexedData& data) {
    const auto names = data.getBlocksOfType<HNS::Vec3f>();
    if (names.size() != 1) throw std::runtime_error("Expected exactly one Vec3f block (velocity)");
    return names[0];
}

// A throwaway context over data's grid on the caller's stream (the SOP-facing operators
// build their grid on every call, as the reference's did).
struct ScopedCtx {
    hns_ctx* c = nullptr;
    cudaStream_t s = nullptr;  // the stream every copy and kernel of the call goes on
    ScopedCtx(const HNS::GridIndexedData& data, float voxelSize, cudaStream_t stream) {
        const std::vector<int32_t> o = leaves_of(data);
        ok(hns_create(&c, o.data(), (int64_t)o.size() / 3, voxelSize, current_device()), "create");
        if (stream) ok(hns_set_stream(c, stream), "set_stream");
        s = static_cast<cudaStream_t>(hns_get_stream(c));
    }
    ~ScopedCtx() {
        if (c) (void)hns_destroy(c);
    }
};

// Device scratch for the SOP-facing operators.
struct DevArray {
    float* p = nullptr;
    explicit DevArray(size_t n) {
        if (cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(float)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    }
    ~DevArray() {
        if (p) (void)cudaFree(p);
    }
};

void upload(float* d, const void* h, size_t count, cudaStream_t s) {
    if (cudaMemcpyAsync(d, h, count * sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess)
        throw std::runtime_error("host to device copy failed");
}

void download(void* h, const float* d, size_t count, cudaStream_t s) {
    if (cudaMemcpyAsync(h, d, count * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        throw std::runtime_error("device to host copy failed");
}

struct Cache {
    std::vector<int32_t> origins;
    float voxelSize = 0.f;
};

}  // namespace

extern "C" {

HNS_API void CreateIndexGrid(HNS::GridIndexedData& data, HNS::IndexGridHandle& handle, float voxelSize) {
    handle.leafOrigins = leaves_of(data);
    handle.voxelSize = voxelSize;
}

HNS_API void HNS_DestroyContext(void** ctx) {
    if (!ctx || !*ctx) return;
    (void)hns_destroy(static_cast<hns_ctx*>(*ctx));
    *ctx = nullptr;
}

HNS_API void HNS_EnsureContext(void** ctx, HNS::GridIndexedData& data, const HNS::IndexGridHandle& handle,
                               float voxelSize, bool hasCollision) {
    if (!ctx) throw std::runtime_error("HNS_EnsureContext: null context pointer");
    const size_t N = data.size();
    if (!N) throw std::runtime_error("HNS_EnsureContext: N==0");
    if (handle.empty()) throw std::runtime_error("HNS_EnsureContext: deviceGrid() returned null");
    if (handle.numVoxels() != N) throw std::runtime_error("HNS_EnsureContext: grid and data sizes differ");
    hns_ctx* C = static_cast<hns_ctx*>(*ctx);
    bool same_topology = false;
    if (C && (size_t)hns_num_voxels(C) == N && hns_voxel_size(C) == voxelSize) {
        std::vector<int32_t> cur(handle.leafOrigins.size());
        ok(hns_leaf_origins(C, cur.data()), "leaf_origins");
        same_topology = cur == handle.leafOrigins;
        if (!same_topology) {
            // The reference swaps in the new grid and keeps the device state; libhns keeps
            // the state and rebuilds the leaf tables around it.
            std::vector<std::pair<std::string, std::vector<float>>> keep;
            const int count = hns_field_count(C);
            for (int q = 0; q < count; ++q) {
                char name[256];
                int comps = 1;
                ok(hns_field_info(C, q, name, sizeof(name), &comps), "field_info");
                std::vector<float> h(N * (size_t)comps);
                ok(hns_field_get(C, name, h.data(), 0), "field_get");
                keep.emplace_back(std::string(name) + (comps == 3 ? "\x01" : ""), std::move(h));
            }
            hns_ctx* n = nullptr;
            ok(hns_create(&n, handle.leafOrigins.data(), (int64_t)handle.leafOrigins.size() / 3, voxelSize, current_device()),
               "create");
            for (auto& kv : keep) {
                const bool v3 = !kv.first.empty() && kv.first.back() == '\x01';
                const std::string name = v3 ? kv.first.substr(0, kv.first.size() - 1) : kv.first;
                ok(hns_field_set(n, name.c_str(), v3 ? 3 : 1, kv.second.data(), 0), "field_set");
            }
            (void)hns_destroy(C);
            *ctx = C = n;
        }
    } else {
        if (C) HNS_DestroyContext(ctx);
        C = nullptr;
        ok(hns_create(&C, handle.leafOrigins.data(), (int64_t)handle.leafOrigins.size() / 3, voxelSize, current_device()),
           "create");
        *ctx = C;
        const std::string vel = velocity_block(data);
        if (vel.empty()) throw std::runtime_error("No Vec3f blocks in feedback");
        ok(hns_field_set(C, "velocity", 3, reinterpret_cast<const float*>(data.pValues<HNS::Vec3f>(vel)), 0), "velocity");
        for (const auto& name : data.getBlocksOfType<float>()) {
            if (name == "collision_sdf" || is_source(name)) continue;
            ok(hns_field_set(C, name.c_str(), 1, data.pValues<float>(name), 0), name.c_str());
        }
    }
    const auto floats = data.getBlocksOfType<float>();
    const bool have_sdf = hasCollision && std::find(floats.begin(), floats.end(), "collision_sdf") != floats.end();
    if (have_sdf) {
        ok(hns_field_set(C, "collision_sdf", 1, data.pValues<float>("collision_sdf"), 0), "collision_sdf");
    } else {
        float* p = nullptr;
        if (hns_field_ptr(C, "collision_sdf", &p, nullptr) == HNS_OK) (void)hns_field_remove(C, "collision_sdf");
    }
}

HNS_API void HNS_UploadSources(void* ctx, HNS::GridIndexedData& data) {
    hns_ctx* C = static_cast<hns_ctx*>(ctx);
    if (!C || hns_num_voxels(C) == 0) return;
    // Reset the per-cook sources.
    std::vector<std::string> old;
    for (int q = 0; q < hns_field_count(C); ++q) {
        char name[256];
        ok(hns_field_info(C, q, name, sizeof(name), nullptr), "field_info");
        if (is_source(name)) old.emplace_back(name);
    }
    for (const auto& n : old) ok(hns_field_remove(C, n.c_str()), "field_remove");
    const auto v3 = data.getBlocksOfType<HNS::Vec3f>();
    if (std::find(v3.begin(), v3.end(), "src_vel") != v3.end()) {
        if (const auto* h = data.pValues<HNS::Vec3f>("src_vel"))
            ok(hns_field_set(C, "src_vel", 3, reinterpret_cast<const float*>(h), 0), "src_vel");
    }
    for (const auto& name : data.getBlocksOfType<float>()) {
        if (!is_source(name)) continue;
        if (const float* h = data.pValues<float>(name)) ok(hns_field_set(C, name.c_str(), 1, h, 0), name.c_str());
    }
}

HNS_API void HNS_Advance(void* ctx, int iteration, float dt, const CombustionParams& params) {
    hns_ctx* C = static_cast<hns_ctx*>(ctx);
    if (!C || hns_num_voxels(C) == 0) return;
    ok(hns_advance(C, iteration, dt, &params), "HNS_Advance");
    ok(hns_synchronize(C), "HNS_Advance");
}

HNS_API void HNS_DownloadForOutput(void* ctx, HNS::GridIndexedData& data) {
    hns_ctx* C = static_cast<hns_ctx*>(ctx);
    if (!C) throw std::runtime_error("HNS_DownloadForOutput: null context");
    const std::string vel = velocity_block(data);
    if (vel.empty()) return;
    ok(hns_field_get(C, "velocity", reinterpret_cast<float*>(data.pValues<HNS::Vec3f>(vel)), 0), "velocity");
    for (int q = 0; q < hns_field_count(C); ++q) {
        char name[256];
        int comps = 0;
        ok(hns_field_info(C, q, name, sizeof(name), &comps), "field_info");
        if (comps != 1 || is_source(name) || std::strcmp(name, "collision_sdf") == 0) continue;
        if (float* h = data.pValues<float>(name)) ok(hns_field_get(C, name, h, 0), name);
    }
}

HNS_API void HNS_GetActiveMask(void* ctx, std::vector<unsigned char>& hostMask) {
    hns_ctx* C = static_cast<hns_ctx*>(ctx);
    if (!C || hns_num_voxels(C) == 0) {
        hostMask.clear();
        return;
    }
    hostMask.resize((size_t)hns_num_voxels(C));
    ok(hns_active_mask(C, hostMask.data()), "active_mask");
}

HNS_API void Compute_Sim(HNS::GridIndexedData&, const HNS::IndexGridHandle&, int, float, float, const CombustionParams&, bool,
                         const cudaStream_t&) {}

HNS_API void AdvectIndexGrid(HNS::GridIndexedData& data, float dt, float voxelSize, const cudaStream_t& stream) {
    const std::string vel = single_velocity_block(data);
    const auto floats = data.getBlocksOfType<float>();
    if (floats.empty()) throw std::runtime_error("No float blocks found");
    const size_t n = data.size();
    ScopedCtx c(data, voxelSize, stream);
    DevArray dv(3 * n), din(n), dout(n);
    upload(dv.p, data.pValues<HNS::Vec3f>(vel), 3 * n, c.s);
    for (const auto& name : floats) {
        float* h = data.pValues<float>(name);
        upload(din.p, h, n, c.s);
        ok(hns_advect_scalar(c.c, dv.p, din.p, dout.p, dt), "AdvectIndexGrid");
        download(h, dout.p, n, c.s);
    }
    ok(hns_synchronize(c.c), "AdvectIndexGrid");
}

HNS_API void AdvectIndexGridVelocity(HNS::GridIndexedData& data, float dt, float voxelSize, const cudaStream_t& stream) {
    const std::string vel = single_velocity_block(data);
    const size_t n = data.size();
    ScopedCtx c(data, voxelSize, stream);
    DevArray dv(3 * n), dout(3 * n);
    float* h = reinterpret_cast<float*>(data.pValues<HNS::Vec3f>(vel));
    upload(dv.p, h, 3 * n, c.s);
    ok(hns_advect_vec3(c.c, dv.p, dout.p, dt), "AdvectIndexGridVelocity");
    download(h, dout.p, 3 * n, c.s);
    ok(hns_synchronize(c.c), "AdvectIndexGridVelocity");
}

HNS_API void ProjectNonDivergent(HNS::GridIndexedData& data, size_t iteration, float voxelSize, const cudaStream_t& stream) {
    const std::string vel = single_velocity_block(data);
    const size_t n = data.size();
    ScopedCtx c(data, voxelSize, stream);
    DevArray dv(3 * n);
    float* h = reinterpret_cast<float*>(data.pValues<HNS::Vec3f>(vel));
    upload(dv.p, h, 3 * n, c.s);
    ok(hns_project(c.c, dv.p, (int)iteration, -1.0f, 0u, nullptr), "ProjectNonDivergent");
    download(h, dv.p, 3 * n, c.s);
    ok(hns_synchronize(c.c), "ProjectNonDivergent");
}

HNS_API void Divergence(HNS::GridIndexedData& data, float voxelSize, const cudaStream_t& stream) {
    const std::string vel = single_velocity_block(data);
    float* hdiv = data.pValues<float>("divergence");
    if (!hdiv) throw std::runtime_error("Divergence: no float block named 'divergence'");
    const size_t n = data.size();
    ScopedCtx c(data, voxelSize, stream);
    DevArray dv(3 * n), dd(n);
    upload(dv.p, data.pValues<HNS::Vec3f>(vel), 3 * n, c.s);
    ok(hns_divergence(c.c, dv.p, dd.p), "Divergence");
    download(hdiv, dd.p, n, c.s);
    ok(hns_synchronize(c.c), "Divergence");
}

}  // extern "C"
