// Drives libhns through the reference's own C++ entry points (include/hns_legacy.hpp) the
// way the reference's SOPs do (src/SOP/HNanoSolver/SOP_HNanoSolver.cpp:291-396 and the
// SOP-facing operators), and writes every input and output as raw float32 files into the
// directory given as argv[1] for tests/test_gpu_legacy.py to check against the oracle.
// Exit status 0 = every call behaved (values are checked by the pytest side).
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "hns_legacy.hpp"

static std::string g_dir;

static void dump(const std::string& name, const void* p, size_t bytes) {
    FILE* f = std::fopen((g_dir + "/" + name).c_str(), "wb");
    if (!f || std::fwrite(p, 1, bytes, f) != bytes) throw std::runtime_error("cannot write " + name);
    std::fclose(f);
}

// A 2x2x2 block of leaves at negative and positive coordinates minus one leaf, with
// deterministic fields.
static void fill(HNS::GridIndexedData& data, bool with_sources) {
    std::vector<HNS::Coord> origins;
    for (int x = -8; x <= 0; x += 8)
        for (int y = -8; y <= 0; y += 8)
            for (int z = 0; z <= 8; z += 8)
                if (!(x == 0 && y == 0 && z == 8)) origins.push_back({x, y, z});
    const size_t n = origins.size() * 512;
    data.allocateCoords(n);
    data.addValueBlock<float>("density", n);
    data.addValueBlock<float>("temperature", n);
    data.addValueBlock<HNS::Vec3f>("velocity", n);
    if (with_sources) {
        data.addValueBlock<float>("src_temperature", n);
        data.addValueBlock<float>("src_fuel", n);
        data.addValueBlock<HNS::Vec3f>("src_vel", n);
    }
    HNS::Coord* c = data.pCoords();
    float* d = data.pValues<float>("density");
    float* t = data.pValues<float>("temperature");
    HNS::Vec3f* v = data.pValues<HNS::Vec3f>("velocity");
    for (size_t l = 0; l < origins.size(); ++l)
        for (int q = 0; q < 512; ++q) {
            const size_t s = l * 512 + (size_t)q;
            c[s] = {origins[l].x + ((q >> 6) & 7), origins[l].y + ((q >> 3) & 7), origins[l].z + (q & 7)};
            const float x = (float)c[s].x, y = (float)c[s].y, z = (float)c[s].z;
            d[s] = 0.5f + 0.5f * std::sin(0.3f * x) * std::cos(0.2f * y + 0.1f * z);
            t[s] = 0.8f * d[s];
            v[s] = {2.0f * std::sin(0.25f * y + 0.1f * z), 2.0f * std::cos(0.2f * x - 0.15f * z), 1.5f * std::sin(0.3f * x + 0.2f * y)};
            if (with_sources) {
                data.pValues<float>("src_temperature")[s] = (q % 7 == 0) ? 2.0f : 0.0f;
                data.pValues<float>("src_fuel")[s] = (q % 5 == 0) ? 1.0f : 0.0f;
                data.pValues<HNS::Vec3f>("src_vel")[s] = {0.0f, (q % 3 == 0) ? 0.5f : 0.0f, 0.0f};
            }
        }
}

static void dump_all(const HNS::GridIndexedData& data, const std::string& prefix) {
    const size_t n = data.size();
    dump(prefix + "coords.i32", data.pCoords(), n * sizeof(HNS::Coord));
    for (const auto& name : data.getBlocksOfType<float>()) dump(prefix + name + ".f32", data.pValues<float>(name), n * 4);
    for (const auto& name : data.getBlocksOfType<HNS::Vec3f>())
        dump(prefix + name + ".v3", data.pValues<HNS::Vec3f>(name), n * 12);
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    g_dir = argv[1];
    try {
        // ---- the HNanoSolver SOP cook, two frames on one cached context ----
        HNS::GridIndexedData data;
        data.setAllocationType(AllocationType::CudaPinned);
        fill(data, true);
        dump_all(data, "in_");
        CombustionParams params{};
        params.expansionRate = 0.1f, params.temperatureRelease = 0.5f, params.buoyancyStrength = 1.0f;
        params.ambientTemp = 0.4f, params.vorticityScale = 0.5f, params.factorScale = 1.0f;
        params.disturbanceEnable = 1.0f, params.substeps = 2, params.gravity = 1.0f, params.downloadVel = 1;
        void* ctx = nullptr;
        HNS::IndexGridHandle handle;
        CreateIndexGrid(data, handle, 0.1f);
        for (int frame = 0; frame < 2; ++frame) {
            HNS_EnsureContext(&ctx, data, handle, 0.1f, false);
            HNS_UploadSources(ctx, data);
            HNS_Advance(ctx, 10, 1.0f / 24.0f, params);
            HNS_DownloadForOutput(ctx, data);
        }
        std::vector<unsigned char> mask;
        HNS_GetActiveMask(ctx, mask);
        if (mask.size() != data.size()) throw std::runtime_error("mask size");
        for (unsigned char m : mask)
            if (m != 1) throw std::runtime_error("mask value");
        dump_all(data, "advance_");
        HNS_DestroyContext(&ctx);
        if (ctx != nullptr) throw std::runtime_error("context not cleared");
        HNS_Advance(ctx, 10, 0.1f, params);  // null context: a no-op, as in the reference

        // ---- the SOP-facing operators: advect scalars, advect velocity, project ----
        HNS::GridIndexedData sop;
        fill(sop, false);
        sop.addValueBlock<float>("divergence", sop.size());
        cudaStream_t stream = nullptr;
        Divergence(sop, 0.1f, stream);
        dump(std::string("sopdiv_divergence.f32"), sop.pValues<float>("divergence"), sop.size() * 4);
        AdvectIndexGrid(sop, 0.1f, 0.1f, stream);  // also advects "divergence": every float block
        AdvectIndexGridVelocity(sop, 0.1f, 0.1f, stream);
        ProjectNonDivergent(sop, 20, 0.1f, stream);
        dump_all(sop, "sop_");

        // ---- error behaviour: exceptions, as the reference's CUDA_CHECK throws ----
        int thrown = 0;
        sop.addValueBlock<HNS::Vec3f>("second_vel", sop.size());
        try {
            AdvectIndexGridVelocity(sop, 0.1f, 0.1f, stream);
        } catch (const std::runtime_error&) {
            ++thrown;
        }
        HNS::GridIndexedData bad;
        bad.allocateCoords(512);
        bad.addValueBlock<HNS::Vec3f>("velocity", 512);
        try {
            HNS::IndexGridHandle h;
            CreateIndexGrid(bad, h, 0.1f);  // all-zero coordinates are not leaf-dense
        } catch (const std::runtime_error&) {
            ++thrown;
        }
        HNS::GridIndexedData empty;
        try {
            void* c2 = nullptr;
            HNS_EnsureContext(&c2, empty, handle, 0.1f, false);
        } catch (const std::runtime_error&) {
            ++thrown;
        }
        if (thrown != 3) throw std::runtime_error("expected three exceptions, saw " + std::to_string(thrown));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "legacy_api_test: %s\n", e.what());
        return 1;
    }
    std::printf("legacy_api_test ok\n");
    return 0;
}
