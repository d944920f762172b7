// Launch driver for the reference's own kernels, compiled as host C++.
//
// TEST INFRASTRUCTURE ONLY. This file is the "oracle/_ref" leg of the oracle: it includes
// the reference's unmodified src/Cuda/Kernel.cu (through oracle/ref_shim/cudashim.h) and
// runs each __global__ function as a loop over (block, thread), with OpenMP across
// blocks. The index grid is the reference's NanoVDB ValueOnIndex grid built on the host
// with the vendored NanoVDB tools. The step sequence of HNS_Advance
// (src/Cuda/HNanoSolver.cu:223-456) and of the SOP-facing operators
// (src/Cuda/Advection.cu:13-166, src/Cuda/PressureProjection.cu:9-129, both commented out
// in the reference) is restated here as host launch loops; the arithmetic is the
// reference's. Only tests/, bench.py's reference arm and the smoke check call it.
#include "cudashim.h"

thread_local hns_shim_uint3 blockIdx;
thread_local hns_shim_uint3 threadIdx;
thread_local hns_shim_uint3 blockDim;

#include "Kernel.cu"  // reference: src/Cuda/Kernel.cu (include path set by oracle/Makefile)

#include <nanovdb/tools/CreateNanoGrid.h>
#include <nanovdb/tools/GridBuilder.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using IndexGrid = nanovdb::NanoGrid<nanovdb::ValueOnIndex>;

struct RefGrid {
    nanovdb::GridHandle<nanovdb::HostBuffer> handle;
    const IndexGrid* grid = nullptr;
};

// Fraction of thread blocks each launch runs: 1 = the whole launch. The CPU baseline
// times a bounded sample of a workload by running every launch of a step over an evenly
// spaced subset of its blocks (per-voxel work is independent inside each launch).
int g_block_stride = 1;

template <typename F>
void launch(size_t total, F&& body) {
    const unsigned threads = 256;  // HNS_Advance launch shape (src/Cuda/HNanoSolver.cu:232-233)
    const long long blocks = (long long)((total + threads - 1) / threads);
    const int stride = g_block_stride;
#pragma omp parallel for schedule(static)
    for (long long b = 0; b < blocks; b += stride) {
        blockIdx = {unsigned(b), 0, 0};
        blockDim = {threads, 1, 1};
        for (unsigned t = 0; t < threads; ++t) {
            threadIdx = {t, 0, 0};
            body();
        }
    }
}

inline const nanovdb::Coord* C(const int32_t* p) { return reinterpret_cast<const nanovdb::Coord*>(p); }
inline const nanovdb::Vec3f* V(const float* p) { return reinterpret_cast<const nanovdb::Vec3f*>(p); }
inline nanovdb::Vec3f* V(float* p) { return reinterpret_cast<nanovdb::Vec3f*>(p); }

}  // namespace

extern "C" {

int ref_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ref_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void ref_set_block_stride(int stride) { g_block_stride = stride < 1 ? 1 : stride; }

// Index grid from voxel coordinates, as CreateIndexGrid does on the device
// (src/Cuda/HNanoSolver.cu:498-510); built here with the host tools the reference's
// tests use (Tests/IndexGrid.cpp:125, tools/CreateNanoGrid.h:165-175).
void* ref_grid_create(const int32_t* coords, int64_t n) {
    nanovdb::tools::build::Grid<float> src(0.0f);
    auto acc = src.getAccessor();
    for (int64_t i = 0; i < n; ++i) acc.setValue(nanovdb::Coord(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]), 1.0f);
    auto* g = new RefGrid();
    g->handle = nanovdb::tools::createNanoGrid<nanovdb::tools::build::Grid<float>, nanovdb::ValueOnIndex>(src, 0u, false, false, 0);
    g->grid = g->handle.grid<nanovdb::ValueOnIndex>();
    return g;
}

void ref_grid_destroy(void* g) { delete static_cast<RefGrid*>(g); }

uint64_t ref_grid_value_count(void* g) { return static_cast<RefGrid*>(g)->grid->valueCount(); }

uint64_t ref_grid_leaf_count(void* g) { return static_cast<RefGrid*>(g)->grid->tree().nodeCount(0); }

// Leaf origins in the grid's own leaf order (the order value offsets are assigned in).
void ref_grid_leaf_origins(void* g, int32_t* out) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    const auto* leaf = grid->tree().getFirstNode<0>();
    const uint64_t count = grid->tree().nodeCount(0);
    for (uint64_t i = 0; i < count; ++i) {
        const nanovdb::Coord o = leaf[i].origin();
        out[3 * i] = o[0];
        out[3 * i + 1] = o[1];
        out[3 * i + 2] = o[2];
    }
}

// NanoVDB ValueOnIndex offsets through the reference's IndexOffsetSampler<0>
// (src/Utils/Stencils.hpp:51-71): 0 = background, else 1 + linear value index.
void ref_grid_offsets(void* g, const int32_t* ijk, int64_t n, uint64_t* out) {
    const IndexOffsetSampler<0> s(static_cast<RefGrid*>(g)->grid);
    for (int64_t i = 0; i < n; ++i) out[i] = s.offset(ijk[3 * i], ijk[3 * i + 1], ijk[3 * i + 2]);
}

// Reference samplers (src/Utils/Stencils.hpp:74-172) at arbitrary points.
void ref_sample_scalar(void* g, const float* data, const float* xyz, int64_t n, int order, float* out) {
    const IndexOffsetSampler<0> s(static_cast<RefGrid*>(g)->grid);
    const IndexSampler<float, 1> tri(s, data);
    const IndexSampler<float, 0> near(s, data);
    for (int64_t i = 0; i < n; ++i) {
        if (order == 0) {
            out[i] = near(nanovdb::Coord((int)xyz[3 * i], (int)xyz[3 * i + 1], (int)xyz[3 * i + 2]));
        } else {
            out[i] = tri(nanovdb::Vec3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
        }
    }
}

void ref_sample_vec3(void* g, const float* data, const float* xyz, int64_t n, int order, float* out) {
    const IndexOffsetSampler<0> s(static_cast<RefGrid*>(g)->grid);
    const IndexSampler<nanovdb::Vec3f, 1> tri(s, V(data));
    const IndexSampler<nanovdb::Vec3f, 0> near(s, V(data));
    for (int64_t i = 0; i < n; ++i) {
        nanovdb::Vec3f v;
        if (order == 0) {
            v = near(nanovdb::Coord((int)xyz[3 * i], (int)xyz[3 * i + 1], (int)xyz[3 * i + 2]));
        } else {
            v = tri(nanovdb::Vec3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
        }
        out[3 * i] = v[0];
        out[3 * i + 1] = v[1];
        out[3 * i + 2] = v[2];
    }
}

// ---- single kernels (Kernel.cu), one launch each ---------------------------------------

void ref_advect_vector(void* g, const int32_t* coords, int64_t n, const float* vel, float* out, float dt, float inv_dx) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { advect_vector(grid, C(coords), V(vel), V(out), nullptr, false, nullptr, (size_t)n, dt, inv_dx); });
}

void ref_advect_scalars(void* g, const int32_t* coords, int64_t n, const float* vel, float** in, float** out, int nfields,
                        float dt, float inv_dx) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { advect_scalars(grid, C(coords), V(vel), in, out, nfields, nullptr, false, nullptr, (size_t)n, dt, inv_dx); });
}

void ref_advect_scalar(void* g, const int32_t* coords, int64_t n, const float* vel, const float* in, float* out, float dt,
                       float inv_dx) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { advect_scalar(grid, C(coords), V(vel), in, out, nullptr, false, (size_t)n, dt, inv_dx, nullptr); });
}

void ref_divergence(void* g, const int32_t* coords, int64_t n, const float* vel, float* div, float inv_dx) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { divergence(grid, C(coords), V(vel), div, inv_dx, nullptr, (size_t)n); });
}

void ref_rbgs(void* g, const int32_t* coords, int64_t n, const float* div, float* p, float dx, int iterations, float omega) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    for (int it = 0; it < iterations; ++it) {
        for (int color = 0; color < 2; ++color) {
            launch(n, [&] { redBlackGaussSeidelUpdate(grid, C(coords), div, p, dx, (size_t)n, color, omega, nullptr); });
        }
    }
}

void ref_subtract_gradient(void* g, const int32_t* coords, int64_t n, const float* vel, const float* p, float* out,
                           float inv_dx) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { subtractPressureGradient(grid, C(coords), (size_t)n, V(vel), p, V(out), nullptr, false, inv_dx, nullptr); });
}

// Out of place: the reference launches it in place (src/Cuda/HNanoSolver.cu:279-281),
// which is a read/write race across threads; the oracle fixes the race-free meaning.
void ref_vorticity_confinement(void* g, const int32_t* coords, int64_t n, const float* vel, float* out, float dt,
                               float inv_dx, float scale, float factor_scale) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    launch(n, [&] { vorticityConfinement(grid, C(coords), V(vel), V(out), dt, inv_dx, scale, factor_scale, nullptr, (size_t)n); });
}

void ref_temperature_buoyancy(int64_t n, const float* vel, const float* temp, float* out, float dt, float ambient,
                              float strength) {
    launch(n, [&] { temperature_buoyancy(V(vel), temp, V(out), dt, ambient, strength, nullptr, (size_t)n); });
}

void ref_combustion(int64_t n, const float* fuel, const float* temp, float* out_fuel, float* out_temp, float dt,
                    float ignition, float rate, float heat) {
    launch(n, [&] { combustion(nullptr, nullptr, fuel, temp, out_fuel, out_temp, dt, ignition, rate, heat, (size_t)n); });
}

void ref_combustion_oxygen(int64_t n, const float* fuel, const float* waste, const float* temp, float* div,
                           const float* flame, float* o_fuel, float* o_waste, float* o_temp, float* o_flame, float gain,
                           float expansion) {
    launch(n, [&] { combustion_oxygen(fuel, waste, temp, div, flame, o_fuel, o_waste, o_temp, o_flame, gain, expansion, nullptr, (int)n); });
}

void ref_add_scalar_source(int64_t n, float* field, const float* src, float dt) {
    launch(n, [&] { add_scalar_source(field, src, dt, nullptr, (int)n); });
}

void ref_add_velocity_source(int64_t n, float* vel, const float* src, float dt) {
    launch(n, [&] { add_velocity_source(V(vel), V(src), dt, nullptr, (int)n); });
}

void ref_add_velocity_source_xyz(int64_t n, float* vel, const float* sx, const float* sy, const float* sz, float dt) {
    launch(n, [&] { add_velocity_source_xyz(V(vel), sx, sy, sz, dt, nullptr, (int)n); });
}

void ref_add_gravity(int64_t n, float* vel, float g, float dt) {
    launch(n, [&] { add_gravity(V(vel), g, dt, nullptr, (int)n); });
}

// ---- operator sequences ------------------------------------------------------------------

// HNanoProjectNonDivergent: divergence, iterations x (red, black) SOR sweeps from p = 0,
// gradient subtraction written back into the velocity (src/Cuda/PressureProjection.cu:9-78).
// omega < 0 selects that path's 2/(1+sin(3.14159*dx)), evaluated in double and stored as
// float (PressureProjection.cu:53).
void ref_project(void* g, const int32_t* coords, int64_t n, float* vel, float* div, float* p, float dx, int iterations,
                 float omega) {
    const float inv_dx = 1.0f / dx;
    if (omega < 0.0f) omega = (float)(2.0f / (1.0f + sin(3.14159 * dx)));
    ref_divergence(g, coords, n, vel, div, inv_dx);
    std::fill(p, p + n, 0.0f);
    ref_rbgs(g, coords, n, div, p, dx, iterations, omega);
    std::vector<float> tmp(vel, vel + 3 * n);
    ref_subtract_gradient(g, coords, n, tmp.data(), p, vel, inv_dx);
}

// One step of the SOP operator chain HNanoAdvect + HNanoAdvectVelocity +
// HNanoProjectNonDivergent with the reference's kernels (the SOP bodies are commented out in
// the reference, src/Cuda/Advection.cu:13-166 and src/Cuda/PressureProjection.cu:9-78): the
// scalars and the velocity are advected with the old velocity, then the velocity is
// projected with `iterations` red-black sweeps from p = 0. `scratch` holds 5n floats.
// With a block stride > 1 (ref_set_block_stride) every launch runs a subset of its blocks:
// the timed CPU baseline's bounded sample.
void ref_plain_step(void* g, const int32_t* coords, int64_t n, float* vel, float* const* scalars, int nscalars, float dt,
                    float dx, int iterations, float omega, float* scratch) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    const float inv_dx = 1.0f / dx;
    float* adv = scratch;          // 3n
    float* div = scratch + 3 * n;  // n
    float* p = scratch + 4 * n;    // n
    std::vector<float> tmp(nscalars > 0 ? n : 0);
    for (int q = 0; q < nscalars; ++q) {
        float* in = scalars[q];
        float* out = tmp.data();
        launch(n, [&] { advect_scalar(grid, C(coords), V(vel), in, out, nullptr, false, (size_t)n, dt, inv_dx, nullptr); });
        std::copy(tmp.begin(), tmp.end(), in);
    }
    launch(n, [&] { advect_vector(grid, C(coords), V(vel), V(adv), nullptr, false, nullptr, (size_t)n, dt, inv_dx); });
    launch(n, [&] { divergence(grid, C(coords), V(adv), div, inv_dx, nullptr, (size_t)n); });
    std::fill(p, p + n, 0.0f);
    ref_rbgs(g, coords, n, div, p, dx, iterations, omega);
    launch(n, [&] { subtractPressureGradient(grid, C(coords), (size_t)n, V(adv), p, V(vel), nullptr, false, inv_dx, nullptr); });
}

// Field set for the HNS_Advance restatement. `names`/`scalars` are the persistent scalar
// fields present when the call starts (the context's d_state, HNanoSolver.cu:113-119):
// exactly these are advected (advNames is taken before the substep loop, :247-250).
// fuel/waste/temperature/flame that are absent from that list are created zero-filled on
// first use (needOrMake, :326-338) in the caller-provided `created` buffers and are not
// advected during this call.
struct RefAdvanceFields {
    int64_t n;
    float* velocity;  // 3n, in/out
    int nscalars;
    const char* const* names;
    float* const* scalars;
    float* created[4];  // fuel, waste, temperature, flame when not in names (n each) or NULL
    const float* src_vel;  // 3n or NULL
    const float* src_vel_x;
    const float* src_vel_y;
    const float* src_vel_z;
    const float* src_temperature;
    const float* src_density;
    const float* src_fuel;
    const float* collision_sdf;  // n, or NULL: no collider
};

static float* find_scalar(const RefAdvanceFields* f, const char* name) {
    for (int i = 0; i < f->nscalars; ++i)
        if (std::strcmp(f->names[i], name) == 0) return f->scalars[i];
    return nullptr;
}

// Restates HNS_Advance (src/Cuda/HNanoSolver.cu:223-456), with the reference's collision
// kernels and branches when F->collision_sdf is set (:241-244, :273-275, :406-414, :438-441).
// combustion: 0 runs combustion_oxygen (the reference's step); 1 runs the reference's
// `combustion` kernel (Kernel.cu:568-588) with burn_rate, heat_release and ignition_temp in its
// place, creating only fuel and temperature when absent, the sequence otherwise unchanged.
// omega > 0 replaces HNS_Advance's 2/(1+sin(3.14159 dx)) in its red-black solves.
void ref_hns_advance_model(void* g, const int32_t* coords, const RefAdvanceFields* F, float dx, int iteration, float dt,
                           const CombustionParams* params, int combustion_model, float burn_rate, float heat_release,
                           float ignition_temp, float omega_override) {
    const IndexGrid* grid = static_cast<RefGrid*>(g)->grid;
    const int64_t N = F->n;
    const float inv_dx = 1.0f / dx;
    const int SUBS = std::max(1, params->substeps);
    const float dt_sub = dt / float(SUBS);
    std::vector<float> adv(3 * N, 0.0f), div(N, 0.0f), p(N, 0.0f), adv2(3 * N);
    std::vector<float> o_fuel(N), o_waste(N), o_temp(N), o_flame(N);
    bool made[4] = {false, false, false, false};
    static const char* special[4] = {"fuel", "waste", "temperature", "flame"};
    const nanovdb::Coord* cc = C(coords);
    const float* sdf = F->collision_sdf;
    const bool hc = sdf != nullptr;
    if (hc) launch(N, [&] { enforceCollisionBoundaries(grid, cc, V(F->velocity), sdf, dx, (size_t)N); });

    for (int s = 0; s < SUBS; ++s) {
        // build_activity_mask writes 1 everywhere (Kernel.cu:75): no masking below.
        launch(N, [&] { advect_vector(grid, cc, V(F->velocity), V(adv.data()), sdf, hc, nullptr, (size_t)N, dt_sub, inv_dx); });
        launch(N, [&] { vorticityConfinement(grid, cc, V(adv.data()), V(adv2.data()), dt_sub, inv_dx, params->vorticityScale, params->factorScale, nullptr, (size_t)N); });
        adv.swap(adv2);
        if (F->src_vel) {
            launch(N, [&] { add_velocity_source(V(adv.data()), V(F->src_vel), dt_sub, nullptr, (int)N); });
        } else if (F->src_vel_x && F->src_vel_y && F->src_vel_z) {
            launch(N, [&] { add_velocity_source_xyz(V(adv.data()), F->src_vel_x, F->src_vel_y, F->src_vel_z, dt_sub, nullptr, (int)N); });
        }
        const struct {
            const float* src;
            const char* dst;
        } pairs[] = {{F->src_temperature, "temperature"}, {F->src_density, "density"}, {F->src_fuel, "fuel"}};
        for (const auto& pr : pairs) {
            float* dst = find_scalar(F, pr.dst);
            if (!dst) {  // a field created earlier in this call counts as present (d_state)
                for (int k = 0; k < 4; ++k)
                    if (made[k] && std::strcmp(special[k], pr.dst) == 0) dst = F->created[k];
            }
            if (pr.src && dst) launch(N, [&] { add_scalar_source(dst, pr.src, dt_sub, nullptr, (int)N); });
        }
        if (params->gravity != 0.0f) launch(N, [&] { add_gravity(V(adv.data()), params->gravity, dt_sub, nullptr, (int)N); });
        launch(N, [&] { divergence(grid, cc, V(adv.data()), div.data(), inv_dx, nullptr, (size_t)N); });

        float* fld[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int k = 0; k < 4; ++k) {
            if (combustion_model == 1 && (k == 1 || k == 3)) continue;
            fld[k] = find_scalar(F, special[k]);
            if (!fld[k]) {
                fld[k] = F->created[k];
                if (!made[k]) {
                    std::fill(fld[k], fld[k] + N, 0.0f);
                    made[k] = true;
                }
            }
        }
        std::fill(o_fuel.begin(), o_fuel.end(), 0.0f);
        std::fill(o_waste.begin(), o_waste.end(), 0.0f);
        std::fill(o_temp.begin(), o_temp.end(), 0.0f);
        std::fill(o_flame.begin(), o_flame.end(), 0.0f);
        if (combustion_model == 1) {
            launch(N, [&] {
                combustion(grid, cc, fld[0], fld[2], o_fuel.data(), o_temp.data(), dt_sub, ignition_temp, burn_rate,
                           heat_release, (size_t)N);
            });
        } else {
            launch(N, [&] {
                combustion_oxygen(fld[0], fld[1], fld[2], div.data(), fld[3], o_fuel.data(), o_waste.data(), o_temp.data(),
                                  o_flame.data(), params->temperatureRelease, params->expansionRate, nullptr, (int)N);
            });
        }
        launch(N, [&] {
            temperature_buoyancy(V(adv.data()), o_temp.data(), V(adv.data()), dt_sub, params->ambientTemp, params->buoyancyStrength,
                                 nullptr, (size_t)N);
        });
        std::copy(o_fuel.begin(), o_fuel.end(), fld[0]);
        std::copy(o_temp.begin(), o_temp.end(), fld[2]);
        if (combustion_model != 1) {
            std::copy(o_waste.begin(), o_waste.end(), fld[1]);
            std::copy(o_flame.begin(), o_flame.end(), fld[3]);
        }

        std::fill(p.begin(), p.end(), 0.0f);
        const float omega = omega_override > 0.0f ? omega_override : 2.0f / (1.0f + sinf(3.14159f * dx));
        ref_rbgs(g, coords, N, div.data(), p.data(), dx, iteration, omega);
        if (params->disturbanceEnable > 0.0f) {
            launch(N, [&] { divergence(grid, cc, V(adv.data()), div.data(), inv_dx, nullptr, (size_t)N); });
            std::fill(p.begin(), p.end(), 0.0f);
            ref_rbgs(g, coords, N, div.data(), p.data(), dx, std::max(2, iteration / 2), omega);
        }
        launch(N, [&] { subtractPressureGradient(grid, cc, (size_t)N, V(adv.data()), p.data(), V(F->velocity), sdf, hc, inv_dx, nullptr); });
        if (hc) launch(N, [&] { enforceCollisionBoundaries(grid, cc, V(F->velocity), sdf, dx, (size_t)N); });

        if (F->nscalars > 0) {
            std::vector<std::vector<float>> outs(F->nscalars, std::vector<float>(N, 0.0f));
            std::vector<float*> ins(F->nscalars), outp(F->nscalars);
            for (int k = 0; k < F->nscalars; ++k) {
                ins[k] = F->scalars[k];
                outp[k] = outs[k].data();
            }
            float** pin = ins.data();
            float** pout = outp.data();
            const int ns = F->nscalars;
            launch(N, [&] { advect_scalars(grid, cc, V(F->velocity), pin, pout, ns, sdf, hc, nullptr, (size_t)N, dt_sub, inv_dx); });
            for (int k = 0; k < F->nscalars; ++k) std::copy(outs[k].begin(), outs[k].end(), F->scalars[k]);
        }
    }
}

void ref_hns_advance(void* g, const int32_t* coords, const RefAdvanceFields* F, float dx, int iteration, float dt,
                     const CombustionParams* params) {
    ref_hns_advance_model(g, coords, F, dx, iteration, dt, params, 0, 0.0f, 0.0f, 0.0f, 0.0f);
}

}  // extern "C"
