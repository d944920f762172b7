// The all-in-one solver step of the HNanoSolver SOP (HNS_Advance,
// src/Cuda/HNanoSolver.cu:223-456) over the context's named fields, and the field store
// that replaces the reference's SimContext maps (src/Cuda/HNanoSolver.cu:27-48).
//
// Per substep the reference runs about 2*iterations + 15 launches, with cudaMalloc'd
// temporaries, memsets and device-to-device copies. Here:
//   advect_fused          velocity -> adv                       (advect_vector)
//   confine_sources       adv -> adv2, + sources, gravity       (vorticityConfinement out of
//                                                                place, add_velocity_source(_xyz),
//                                                                add_scalar_source, add_gravity)
//   div_combust_buoy      adv2 -> div, fields, adv3             (divergence, combustion_oxygen or
//                                                                the force model's burn,
//                                                                temperature_buoyancy [+ density])
//   rbgs x iterations     div -> p                              (redBlackGaussSeidelUpdate)
//   [divergence, rbgs x max(2, iterations/2)]  when disturbanceEnable > 0
//   subtract_gradient     adv3, p -> velocity
//   advect_scalars        the persistent scalars, with the projected velocity
// With a "collision_sdf" field the collider enters as in the reference: enforced on the
// velocity before the substeps and after each projection, trace points inside it pulled back
// in both advections, and the near-wall blend after the velocity advection and the gradient.
// Each fusion applies the reference's per-voxel operations in the reference's order, so
// every output equals the reference's (the confinement race aside: it runs out of place).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hns_confine.cuh"
#include "hns_internal.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

using namespace dev;

constexpr int kThreads = 256;

struct ScalarSources {
    float* dst[3];
    const float* src[3];
    int count;
};

// vorticityConfinement (src/Cuda/Kernel.cu:682-727) out of place, then the velocity source
// (add_velocity_source / add_velocity_source_xyz, Kernel.cu:739-755), gravity (add_gravity,
// Kernel.cu:834-838) and the scalar sources (add_scalar_source, Kernel.cu:732-737), in the
// order HNS_Advance launches them (src/Cuda/HNanoSolver.cu:279-318).
__global__ void __launch_bounds__(kThreads) confine_sources_kernel(TopoView t, const float* __restrict__ vel,
                                                                    float* __restrict__ out, float dt, float inv_dx,
                                                                    float scale, int fs, const float* __restrict__ src_v3,
                                                                    const float* __restrict__ sx, const float* __restrict__ sy,
                                                                    const float* __restrict__ sz, float gravity,
                                                                    ScalarSources ss) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float factor = 0.5f * inv_dx;
    const float3 px = near_v(t, L, vel, i + 1, j, k), mx = near_v(t, L, vel, i - 1, j, k);
    const float3 py = near_v(t, L, vel, i, j + 1, k), my = near_v(t, L, vel, i, j - 1, k);
    const float3 pz = near_v(t, L, vel, i, j, k + 1), mz = near_v(t, L, vel, i, j, k - 1);
    const float ox = ((py.z - my.z) - (pz.y - mz.y)) * factor;
    const float oy = ((pz.x - mz.x) - (px.z - mx.z)) * factor;
    const float oz = ((px.y - mx.y) - (py.x - my.x)) * factor;
    const float mpx = vort_mag(t, L, vel, i + fs, j, k, factor), mmx = vort_mag(t, L, vel, i - fs, j, k, factor);
    const float mpy = vort_mag(t, L, vel, i, j + fs, k, factor), mmy = vort_mag(t, L, vel, i, j - fs, k, factor);
    const float mpz = vort_mag(t, L, vel, i, j, k + fs, factor), mmz = vort_mag(t, L, vel, i, j, k - fs, factor);
    const float gx = (mpx - mmx) * 0.5f * inv_dx;
    const float gy = (mpy - mmy) * 0.5f * inv_dx;
    const float gz = (mpz - mmz) * 0.5f * inv_dx;
    const float glen = sqrtf(gx * gx + gy * gy + gz * gz) + 1e-5f;
    const float nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const float3 u = ld3(vel, s);
    const float fx = scale * (ny * oz - nz * oy), fy = scale * (nz * ox - nx * oz), fz = scale * (nx * oy - ny * ox);
    float3 r = make_float3(u.x + fx * dt, u.y + fy * dt, u.z + fz * dt);
    if (src_v3 != nullptr) {
        const float3 a = ld3(src_v3, s);
        r.x += a.x * dt;
        r.y += a.y * dt;
        r.z += a.z * dt;
    } else if (sx != nullptr && sy != nullptr && sz != nullptr) {
        r.x += dt * __ldg(sx + s);
        r.y += dt * __ldg(sy + s);
        r.z += dt * __ldg(sz + s);
    }
    if (gravity != 0.0f) r.y -= gravity * dt;
    st3(out, s, r);
    for (int q = 0; q < ss.count; ++q) ss.dst[q][s] += dt * __ldg(ss.src[q] + s);
}

// confine_sources_kernel on a shared-memory leaf tile (hns_confine.cuh), for |fs| <= 1: one CTA
// per leaf, the same values.
__global__ void __launch_bounds__(kThreads) confine_sources_tile_kernel(TopoView t, const float* __restrict__ vel,
                                                                         float* __restrict__ out, float dt, float inv_dx,
                                                                         float scale, int fs,
                                                                         const float* __restrict__ src_v3,
                                                                         const float* __restrict__ sx,
                                                                         const float* __restrict__ sy,
                                                                         const float* __restrict__ sz, float gravity,
                                                                         ScalarSources ss) {
    __shared__ LeafNbhd L;
    __shared__ ConfineTile T;
    const int64_t leaf = blockIdx.x;
    load_nbhd(L, t, leaf);
    __syncthreads();
    confine_tile(L, vel, T, 0.5f * inv_dx);
    for (int n = threadIdx.x; n < 512; n += blockDim.x) {
        const int64_t s = (leaf << 9) + n;
        float3 r = confine_at(T, n >> 6, (n >> 3) & 7, n & 7, fs, inv_dx, dt, scale);
        if (src_v3 != nullptr) {
            const float3 a = ld3(src_v3, s);
            r.x += a.x * dt;
            r.y += a.y * dt;
            r.z += a.z * dt;
        } else if (sx != nullptr && sy != nullptr && sz != nullptr) {
            r.x += dt * __ldg(sx + s);
            r.y += dt * __ldg(sy + s);
            r.z += dt * __ldg(sz + s);
        }
        if (gravity != 0.0f) r.y -= gravity * dt;
        st3(out, s, r);
        for (int q = 0; q < ss.count; ++q) ss.dst[q][s] += dt * __ldg(ss.src[q] + s);
    }
}

// The burn model and the buoyancy's density term of one step (hns_force_model), with the
// reference's parameters.
struct Burn {
    float gain, expansion;           // combustion_oxygen: temperatureRelease, expansionRate
    float rate, heat, ignition;      // combustion: burn rate, heat release, ignition temperature
    float alpha;                     // density buoyancy; 0: the reference's temperature_buoyancy
};

// divergence (Kernel.cu:432-453) of the forced velocity, the combustion model in place on its
// fields (kModel: HNS_COMBUSTION_OXYGEN, combustion_oxygen (Kernel.cu:641-677) on fuel, waste,
// temperature and flame, the expansion added to that divergence; HNS_COMBUSTION_RATE,
// combustion (Kernel.cu:568-588) on fuel and temperature; HNS_COMBUSTION_NONE), then
// temperature_buoyancy (Kernel.cu:546-563) from the burned temperature, with the density term
// v.y -= alpha density dt when alpha != 0, into a separate velocity buffer (neighbouring
// threads still read `vel`).
template <int kModel>
__global__ void __launch_bounds__(kThreads) div_combust_buoy_kernel(TopoView t, const float* __restrict__ vel,
                                                                     float* __restrict__ vel_out, float* __restrict__ div,
                                                                     float inv_dx, float* __restrict__ fuel,
                                                                     float* __restrict__ waste, float* __restrict__ temp,
                                                                     float* __restrict__ flame,
                                                                     const float* __restrict__ density, Burn B, float dt,
                                                                     float ambient, float strength) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 c = ld3(vel, s);
    const float xp = (c.x + near_v(t, L, vel, i + 1, j, k).x) * 0.5f;
    const float xm = (c.x + near_v(t, L, vel, i - 1, j, k).x) * 0.5f;
    const float yp = (c.y + near_v(t, L, vel, i, j + 1, k).y) * 0.5f;
    const float ym = (c.y + near_v(t, L, vel, i, j - 1, k).y) * 0.5f;
    const float zp = (c.z + near_v(t, L, vel, i, j, k + 1).z) * 0.5f;
    const float zm = (c.z + near_v(t, L, vel, i, j, k - 1).z) * 0.5f;
    float dv = (xp - xm + yp - ym + zp - zm) * inv_dx;

    float Tn = temp[s];
    if constexpr (kModel == HNS_COMBUSTION_OXYGEN) {
        float f = fuel[s];
        const float w = waste[s], T = Tn, fl = flame[s];
        if (f < 0.001f) f = 0.0f;
        const float oxy = 1.0f - f - w;
        if (oxy < 0.0f) {
            fuel[s] = f;
        } else {
            const float burn = fminf(oxy, f);
            fuel[s] = f - burn;
            waste[s] = w + burn * 2.0f;
            Tn = T + burn * B.gain;
            temp[s] = Tn;
            dv += burn * B.expansion;
            flame[s] = fmaxf(fl, fminf(1.0f, burn * 10.0f));
        }
    } else if constexpr (kModel == HNS_COMBUSTION_RATE) {
        const float f = fuel[s];
        if (f > 0.0f && Tn >= B.ignition) {
            const float burned = fminf(f, B.rate * dt);
            fuel[s] = f - burned;
            Tn = Tn + burned * B.heat;
            temp[s] = Tn;
        }
    }
    div[s] = dv;
    if (B.alpha != 0.0f) {
        const float bt = Tn > ambient ? fmaxf(0.0f, (Tn - ambient) * strength) : 0.0f;
        const float fy = bt - B.alpha * (density != nullptr ? __ldg(density + s) : 0.0f);
        st3(vel_out, s, make_float3(c.x, c.y + fy * dt, c.z));
    } else if (Tn <= ambient) {
        st3(vel_out, s, c);
    } else {
        const float by = fmaxf(0.0f, (Tn - ambient) * strength);
        st3(vel_out, s, make_float3(c.x + 0.0f * dt, c.y + by * dt, c.z + 0.0f * dt));
    }
}

unsigned leaf_blocks(const Context& c) { return (unsigned)(c.topo.num_leaves * 2); }

}  // namespace

void launch_div_combust_buoy(const Context& c, const float* vel, float* vel_out, float* div, float* fuel, float* waste,
                             float* temp, float* flame, const float* density, const hns_combustion_params& P,
                             const hns_force_model& M, float dt) {
    const Burn B{P.temperatureRelease, P.expansionRate, M.burn_rate, M.heat_release, M.ignition_temp, M.density_buoyancy};
    const float inv_dx = 1.0f / c.dx;
    if (M.combustion == HNS_COMBUSTION_OXYGEN)
        div_combust_buoy_kernel<HNS_COMBUSTION_OXYGEN><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, vel, vel_out, div, inv_dx, fuel, waste, temp, flame, density, B, dt, P.ambientTemp,
            P.buoyancyStrength);
    else if (M.combustion == HNS_COMBUSTION_RATE)
        div_combust_buoy_kernel<HNS_COMBUSTION_RATE><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, vel, vel_out, div, inv_dx, fuel, waste, temp, flame, density, B, dt, P.ambientTemp,
            P.buoyancyStrength);
    else
        div_combust_buoy_kernel<HNS_COMBUSTION_NONE><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
            c.topo.view, vel, vel_out, div, inv_dx, fuel, waste, temp, flame, density, B, dt, P.ambientTemp,
            P.buoyancyStrength);
    HNS_LAUNCHED();
}

void launch_confine_sources(const Context& c, const float* vel, float* out, float dt, float scale, float factor_scale,
                            const float* src_v3, float gravity) {
    const int fs = (int)factor_scale;
    if (fs >= -1 && fs <= 1)
        confine_sources_tile_kernel<<<(unsigned)c.topo.num_leaves, kThreads, 0, c.stream>>>(
            c.topo.view, vel, out, dt, 1.0f / c.dx, scale, fs, src_v3, nullptr, nullptr, nullptr, gravity, ScalarSources{});
    else
        confine_sources_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(c.topo.view, vel, out, dt, 1.0f / c.dx, scale, fs,
                                                                           src_v3, nullptr, nullptr, nullptr, gravity,
                                                                           ScalarSources{});
    HNS_LAUNCHED();
}

void check_force_model(const hns_force_model& m) {
    if (m.combustion != HNS_COMBUSTION_OXYGEN && m.combustion != HNS_COMBUSTION_RATE && m.combustion != HNS_COMBUSTION_NONE)
        fail(HNS_ERR_INVALID_ARG, "unknown combustion model " + std::to_string(m.combustion));
    if (!std::isfinite(m.burn_rate) || !std::isfinite(m.heat_release) || !std::isfinite(m.ignition_temp) ||
        !std::isfinite(m.density_buoyancy))
        fail(HNS_ERR_INVALID_ARG, "force model parameters must be finite");
}

namespace {

bool is_source(const std::string& n) { return n.rfind("src_", 0) == 0; }

}  // namespace

// ---- field store -----------------------------------------------------------------------------

Field* Context::find_field(const std::string& name) {
    for (auto& f : fields)
        if (f.name == name) return &f;
    return nullptr;
}

Field& Context::ensure_field(const std::string& name, int components, bool zero) {
    Field* f = find_field(name);
    if (f && f->components != components) fail(HNS_ERR_INVALID_ARG, "field '" + name + "' exists with another component count");
    if (!f) {
        fields.push_back(Field{name, components, DeviceBuffer()});
        f = &fields.back();
        f->buf.alloc(sizeof(float) * (size_t)components * (size_t)num_voxels());
        if (zero) HNS_CUDA(cudaMemsetAsync(f->buf.ptr, 0, f->buf.bytes, stream));
    }
    return *f;
}

void run_advance(Context& c, int iterations, float dt, const hns_combustion_params& P, const hns_force_model& M,
                 const hns_step_desc* solve, hns_solve_info* info) {
    const size_t n = (size_t)c.num_voxels();
    const float dx = c.dx;
    const float inv_dx = 1.0f / dx;
    const int subs = std::max(1, P.substeps);
    const float dt_sub = dt / (float)subs;

    // Velocity: "velocity", else the first vec3 field (src/Cuda/HNanoSolver.cu:99-108).
    Field* velf = c.find_field("velocity");
    if (!velf || velf->components != 3) {
        velf = nullptr;
        for (auto& f : c.fields)
            if (f.components == 3 && !is_source(f.name)) {
                velf = &f;
                break;
            }
    }
    if (!velf) fail(HNS_ERR_NOT_FOUND, "no vec3 velocity field in the context");
    const std::string vel_name = velf->name;
    // Persistent scalars present when the call starts are the ones advected (:247-250).
    std::vector<std::string> adv_names;
    for (auto& f : c.fields)
        if (f.components == 1 && !is_source(f.name) && f.name != "collision_sdf") adv_names.push_back(f.name);

    float* adv = c.scratch_f32("advance_adv", 3 * n);
    float* adv2 = c.scratch_f32("advance_adv2", 3 * n);
    float* adv3 = c.scratch_f32("advance_adv3", 3 * n);
    float* div = c.scratch_f32("advance_div", n);
    float* p = c.scratch_f32("advance_p", n);
    const float omega = 2.0f / (1.0f + sinf(3.14159f * dx));  // host sinf, as :365
    const float solve_omega = (solve != nullptr && solve->omega > 0.f) ? solve->omega : omega;
    // A collider: the "collision_sdf" field (HNS_EnsureContext stores it when the SOP has one,
    // :121-133), enforced on the velocity before the substeps (:241-244).
    Field* sdff = c.find_field("collision_sdf");
    const float* sdf = (sdff && sdff->components == 1) ? sdff->buf.as<float>() : nullptr;
    if (sdf && solve != nullptr && (solve->flags & HNS_SOLVE_REFINE))
        fail(HNS_ERR_UNSUPPORTED, "the refined solve of the step does not take a collider");
    if (sdf) launch_collision_enforce(c, c.find_field(vel_name)->buf.as<float>(), sdf);

    for (int s = 0; s < subs; ++s) {
        float* vel = c.find_field(vel_name)->buf.as<float>();
        c.phase_begin(HNS_PHASE_ADVECT);
        FieldSet none{};
        launch_advect_fused(c, vel, adv, none, dt_sub, sdf);
        c.phase_end();

        Field* sv = c.find_field("src_vel");
        Field* sx = c.find_field("src_vel_x");
        Field* sy = c.find_field("src_vel_y");
        Field* sz = c.find_field("src_vel_z");
        ScalarSources ss{};
        static const char* pairs[3][2] = {{"src_temperature", "temperature"}, {"src_density", "density"}, {"src_fuel", "fuel"}};
        for (auto& pr : pairs) {
            Field* src = c.find_field(pr[0]);
            Field* dst = c.find_field(pr[1]);
            if (src && dst && src->components == 1 && dst->components == 1) {
                ss.src[ss.count] = src->buf.as<float>();
                ss.dst[ss.count] = dst->buf.as<float>();
                ++ss.count;
            }
        }
        c.phase_begin(HNS_PHASE_FORCES);
        const float* sv3 = (sv && sv->components == 3) ? sv->buf.as<float>() : nullptr;
        const float* svx = (sx && sx->components == 1) ? sx->buf.as<float>() : nullptr;
        const float* svy = (sy && sy->components == 1) ? sy->buf.as<float>() : nullptr;
        const float* svz = (sz && sz->components == 1) ? sz->buf.as<float>() : nullptr;
        const int fs = (int)P.factorScale;
        if (fs >= -1 && fs <= 1)
            confine_sources_tile_kernel<<<(unsigned)c.topo.num_leaves, kThreads, 0, c.stream>>>(
                c.topo.view, adv, adv2, dt_sub, inv_dx, P.vorticityScale, fs, sv3, svx, svy, svz, P.gravity, ss);
        else
            confine_sources_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, adv, adv2, dt_sub, inv_dx, P.vorticityScale, fs, sv3, svx, svy, svz, P.gravity, ss);
        HNS_LAUNCHED();

        // The combustion model's fields are created zero-filled on first use (:326-338 for
        // the reference's fuel/waste/temperature/flame; fuel and temperature for the rate model,
        // temperature alone without combustion); density when the buoyancy has a density term.
        const bool oxygen = M.combustion == HNS_COMBUSTION_OXYGEN;
        float* fuel = M.combustion != HNS_COMBUSTION_NONE ? c.ensure_field("fuel", 1, true).buf.as<float>() : nullptr;
        float* waste = oxygen ? c.ensure_field("waste", 1, true).buf.as<float>() : nullptr;
        float* temp = c.ensure_field("temperature", 1, true).buf.as<float>();
        float* flame = oxygen ? c.ensure_field("flame", 1, true).buf.as<float>() : nullptr;
        const float* dens = M.density_buoyancy != 0.0f ? c.ensure_field("density", 1, true).buf.as<float>() : nullptr;
        launch_div_combust_buoy(c, adv2, adv3, div, fuel, waste, temp, flame, dens, P, M, dt_sub);
        c.phase_end();

        c.phase_begin(HNS_PHASE_SOLVE);
        const bool refined = solve != nullptr && (solve->flags & HNS_SOLVE_REFINE);
        double* p64 = refined ? reinterpret_cast<double*>(c.scratch_f32("refine_p", 2 * n)) : nullptr;
        // The solve: `iterations` red-black iterations (the reference), or the step
        // description's solve to its tolerance (checked red-black SOR, or the FP32 refinement).
        auto pressure_solve = [&](int its) {
            if (solve == nullptr) {
                rbgs_solve(c, div, p, its, omega, HNS_SOLVE_ZERO_INIT);
            } else if (refined) {
                c.last_refine = refine_solve<float>(c, div, p64, solve->max_outer > 0 ? solve->max_outer : 8,
                                                    solve->inner_iterations > 0 ? solve->inner_iterations : 60,
                                                    solve_omega, solve->tolerance, solve->flags);
            } else {
                c.last_solve = rbgs_solve_checked(c, div, p, solve->max_iterations, solve_omega, HNS_SOLVE_ZERO_INIT,
                                                  solve->tolerance, solve->check_every);
            }
        };
        pressure_solve(iterations);
        if (P.disturbanceEnable > 0.0f) {
            // The disturbance injection is commented out in the reference; what remains is a
            // second, shorter solve of the divergence without the expansion (:377-403).
            launch_divergence(c, adv3, div);
            pressure_solve(std::max(2, iterations / 2));
        }
        c.phase_end();
        c.phase_begin(HNS_PHASE_GRADIENT);
        if (refined) {
            // u = adv3 - grad p with the FP64 pressure, in place on adv3, whose buffer then
            // becomes the velocity field's (the old velocity buffer is the next adv3).
            DeviceBuffer& a3 = c.scratch["advance_adv3"];
            Field* vf = c.find_field(vel_name);
            if (a3.bytes != vf->buf.bytes) fail(HNS_ERR_CUDA, "velocity and step buffers differ in size");
            launch_gradient_f64(c, adv3, p64);
            std::swap(vf->buf, a3);
            adv3 = a3.as<float>();
            vel = vf->buf.as<float>();
        } else {
            vel = c.find_field(vel_name)->buf.as<float>();
            launch_subtract_gradient(c, adv3, p, vel, sdf);
            if (sdf) launch_collision_enforce(c, vel, sdf);  // :411-414
        }
        c.phase_end();

        if (!adv_names.empty()) {
            c.phase_begin(HNS_PHASE_ADVECT);
            // Each field has a twin buffer in the scratch store: the advection writes the twin
            // and the two are swapped, so no step allocates or copies.
            for (size_t base = 0; base < adv_names.size(); base += kMaxAdvectFields) {
                FieldSet f{};
                f.count = (int)std::min<size_t>(kMaxAdvectFields, adv_names.size() - base);
                for (int q = 0; q < f.count; ++q) {
                    f.in[q] = c.find_field(adv_names[base + q])->buf.as<float>();
                    f.out[q] = c.scratch_f32("advance_twin:" + adv_names[base + q], n);
                }
                launch_advect_scalars(c, vel, f, dt_sub, sdf);
            }
            for (const auto& name : adv_names) std::swap(c.find_field(name)->buf, c.scratch["advance_twin:" + name]);
            c.phase_end();
        }
    }
    if (info && solve != nullptr) {
        // The last solve of the call (the one whose pressure made the velocity).
        int its = 0;
        double res = 0.0;
        if (solve->flags & HNS_SOLVE_REFINE) {
            refine_result(c, c.last_refine, &its, &res);
            its *= c.last_refine.inner;
        } else {
            solve_result(c, c.last_solve, &its, &res);
        }
        info->iterations = its;
        info->residual = res;
        info->initial_residual = 1.0;
    }
}

}  // namespace hns

using namespace hns;

extern "C" {

HNS_API hns_status hns_field_set(hns_ctx* ctx, const char* name, int components, const float* data, int on_device) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!name || !*name) fail(HNS_ERR_INVALID_ARG, "empty field name");
        if (components != 1 && components != 3) fail(HNS_ERR_INVALID_ARG, "components must be 1 or 3");
        DeviceGuard g(c->device);
        Field* f = c->find_field(name);
        if (f && f->components != components) {
            c->fields.erase(c->fields.begin() + (f - c->fields.data()));
            f = nullptr;
        }
        Field& fld = c->ensure_field(name, components, data == nullptr);
        if (data && on_device)
            HNS_CUDA(cudaMemcpyAsync(fld.buf.ptr, data, fld.buf.bytes, cudaMemcpyDeviceToDevice, c->stream));
        else if (data)
            copy_h2d(*c, fld.buf.ptr, data, fld.buf.bytes);  // pinned staging; the host buffer may be reused on return
        else
            HNS_CUDA(cudaStreamSynchronize(c->stream));
    });
}

HNS_API hns_status hns_field_get(hns_ctx* ctx, const char* name, float* out, int on_device) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!name || !out) fail(HNS_ERR_INVALID_ARG, "null argument");
        Field* f = c->find_field(name);
        if (!f) fail(HNS_ERR_NOT_FOUND, std::string("no field '") + name + "'");
        DeviceGuard g(c->device);
        if (on_device)
            HNS_CUDA(cudaMemcpyAsync(out, f->buf.ptr, f->buf.bytes, cudaMemcpyDeviceToDevice, c->stream));
        else
            copy_d2h(*c, out, f->buf.ptr, f->buf.bytes);  // pinned staging
    });
}

HNS_API hns_status hns_field_ptr(hns_ctx* ctx, const char* name, float** dev_ptr, int* components) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!name || !dev_ptr) fail(HNS_ERR_INVALID_ARG, "null argument");
        Field* f = c->find_field(name);
        if (!f) fail(HNS_ERR_NOT_FOUND, std::string("no field '") + name + "'");
        *dev_ptr = f->buf.as<float>();
        if (components) *components = f->components;
    });
}

HNS_API hns_status hns_field_remove(hns_ctx* ctx, const char* name) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!name) fail(HNS_ERR_INVALID_ARG, "null name");
        Field* f = c->find_field(name);
        if (!f) fail(HNS_ERR_NOT_FOUND, std::string("no field '") + name + "'");
        DeviceGuard g(c->device);
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        c->fields.erase(c->fields.begin() + (f - c->fields.data()));
    });
}

HNS_API int hns_field_count(const hns_ctx* ctx) { return ctx ? (int)ctx->impl.fields.size() : 0; }

HNS_API hns_status hns_field_info(const hns_ctx* ctx, int index, char* name, size_t name_len, int* components) {
    return guarded([&] {
        const Context* c = check_ctx(ctx);
        if (index < 0 || index >= (int)c->fields.size()) fail(HNS_ERR_INVALID_ARG, "field index out of range");
        const Field& f = c->fields[(size_t)index];
        if (name && name_len > 0) {
            const size_t m = std::min(name_len - 1, f.name.size());
            std::memcpy(name, f.name.data(), m);
            name[m] = '\0';
        }
        if (components) *components = f.components;
    });
}

HNS_API hns_status hns_advance(hns_ctx* ctx, int iterations, float dt, const hns_combustion_params* params) {
    return hns_advance_model(ctx, iterations, dt, params, nullptr);
}

HNS_API hns_status hns_advance_model(hns_ctx* ctx, int iterations, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!params) fail(HNS_ERR_INVALID_ARG, "null params");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        const hns_force_model M = model ? *model : hns_force_model{};
        check_force_model(M);
        DeviceGuard g(c->device);
        run_advance(*c, iterations, dt, *params, M, nullptr, nullptr);
    });
}

HNS_API hns_status hns_advance_solve(hns_ctx* ctx, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model, const hns_step_desc* solve, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        if (!params || !solve) fail(HNS_ERR_INVALID_ARG, "null params or solve description");
        if (!(solve->tolerance > 0.0) || !std::isfinite(solve->tolerance))
            fail(HNS_ERR_INVALID_ARG, "the solve needs a positive tolerance");
        if (!(solve->flags & HNS_SOLVE_REFINE) && solve->max_iterations <= 0)
            fail(HNS_ERR_INVALID_ARG, "the solve needs a positive iteration cap");
        if (solve->flags & ~(unsigned)(HNS_SOLVE_REFINE | HNS_SOLVE_ZERO_INIT))
            fail(HNS_ERR_UNSUPPORTED, "solve flags other than HNS_SOLVE_REFINE are not supported by this step");
        const hns_force_model M = model ? *model : hns_force_model{};
        check_force_model(M);
        DeviceGuard dg(c->device);
        run_advance(*c, 0, dt, *params, M, solve, info);
        if (info && info->residual > solve->tolerance)
            st = record_error(HNS_ERR_NOT_CONVERGED, "pressure solve stopped after " + std::to_string(info->iterations) +
                                                         " iterations with residual " + std::to_string(info->residual));
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_active_mask(hns_ctx* ctx, unsigned char* out) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!out) fail(HNS_ERR_INVALID_ARG, "null output");
        // build_activity_mask writes 1 for every slot (src/Cuda/Kernel.cu:75).
        std::memset(out, 1, (size_t)c->num_voxels());
    });
}

}  // extern "C"
