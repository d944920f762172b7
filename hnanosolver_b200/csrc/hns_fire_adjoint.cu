// Adjoint of the fire step: HNS_Advance (src/Cuda/HNanoSolver.cu:252-452) with a force model,
// one substep, no disturbance re-solve, no collider. Reverse mode through
//   adv  = advect_vector(vel)                            (Kernel.cu:349-426)
//   adv2 = confinement(adv) + dt src_vel + gravity       (Kernel.cu:682-727, 739-745, 834-838)
//   s1   = s + dt src for temperature, density, fuel     (Kernel.cu:732-737)
//   div  = divergence(adv2) [+ expansion burn]           (Kernel.cu:432-453, 641-677)
//   s2   = burn(s1)                                      (Kernel.cu:568-588 or 641-677)
//   adv3 = adv2 + e_y (b_T(T2) - alpha D1) dt            (Kernel.cu:546-563, plus the density term)
//   vel' = adv3 - grad p, p = M div                      (Kernel.cu:459-541)
//   s'   = advect_scalars(vel', s2)                      (Kernel.cu:163-289)
// with the forward recomputed from the step's inputs. M is the step's solve: `iterations`
// red-black iterations from p = 0 (hns_advance_model), whose transpose is the transposed sweeps
// in reverse; or a solve run to a tolerance (hns_advance_mixed), taken as exact: p = L^-1 (dx^2
// div), and L is symmetric, so div_bar = dx^2 L^-1 p_bar is one more refined solve.
//
// As for the other adjoints, branches (the MacCormack clamp, trace cells, the burn's min and
// thresholds, the buoyancy's T > ambient) are frozen at the forward's values, out-of-domain taps
// of advect_scalars read slot 0 (so their adjoint lands on slot 0, as the forward read it), and
// the trilinear scatters use FP32 atomics.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "hns_internal.cuh"
#include "hns_stencil.cuh"

namespace hns {
namespace {

constexpr int kThreads = 256;
constexpr int kFields = 5;  // density, temperature, fuel, waste, flame
enum { kD = 0, kT = 1, kF = 2, kW = 3, kFL = 4 };

unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void coords_at(const TopoView& t, int64_t s, int& i, int& j, int& k) {
    const int4 o = t.origin[s >> 9];
    const int n = (int)(s & 511);
    i = o.x + ((n >> 6) & 7);
    j = o.y + ((n >> 3) & 7);
    k = o.z + (n & 7);
}

// Slot of (i, j, k), with the multi-field advection's fallback: slot 0 outside the domain.
__device__ __forceinline__ int64_t slot0(const TopoView& t, int i, int j, int k) {
    const int s = dev::leaf_from_table(t, i, j, k);
    return s < 0 ? 0 : ((int64_t)s << 9) + dev::local_offset(i, j, k);
}

// setupInterpolation (src/Cuda/Kernel.cu:204-233) as the forward computes it (x fastest in the
// tap index, the same weight products), with the weights' position derivatives.
struct WTaps {
    int64_t s[8];
    float w[8], gx[8], gy[8], gz[8];
};

__device__ __forceinline__ void wtaps(const TopoView& t, float x, float y, float z, WTaps& T) {
    const int i0 = __float2int_rd(x), j0 = __float2int_rd(y), k0 = __float2int_rd(z);
    const float tx = x - (float)i0, ty = y - (float)j0, tz = z - (float)k0;
    const float itx = 1.0f - tx, ity = 1.0f - ty, itz = 1.0f - tz;
    const float w00 = itx * ity, w10 = tx * ity, w01 = itx * ty, w11 = tx * ty;
    T.w[0] = w00 * itz, T.w[1] = w10 * itz, T.w[2] = w01 * itz, T.w[3] = w11 * itz;
    T.w[4] = w00 * tz, T.w[5] = w10 * tz, T.w[6] = w01 * tz, T.w[7] = w11 * tz;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int a = q & 1, b = (q >> 1) & 1, c = (q >> 2) & 1;
        const float wx = a ? tx : itx, wy = b ? ty : ity, wz = c ? tz : itz;
        T.gx[q] = (a ? 1.f : -1.f) * wy * wz;
        T.gy[q] = wx * (b ? 1.f : -1.f) * wz;
        T.gz[q] = wx * wy * (c ? 1.f : -1.f);
        T.s[q] = slot0(t, i0 + a, j0 + b, k0 + c);
    }
}

// Adjoint of advect_scalars for one field d advected along vel (the projected velocity):
// d_bar += (d out / d d)^T out_bar, vel_bar += (d out / d vel)^T out_bar.
__global__ void __launch_bounds__(kThreads) adj_advect_scalars_kernel(TopoView t, const float* __restrict__ vel,
                                                                      const float* __restrict__ d,
                                                                      const float* __restrict__ out_bar,
                                                                      float* __restrict__ d_bar,
                                                                      float* __restrict__ vel_bar, float sdt, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    const float ob = __ldg(out_bar + s);
    if (ob == 0.f) return;
    int i, j, k;
    coords_at(t, s, i, j, k);
    const float3 vc = make_float3(__ldg(vel + 3 * s), __ldg(vel + 3 * s + 1), __ldg(vel + 3 * s + 2));
    const float bx = (float)i - vc.x * sdt, by = (float)j - vc.y * sdt, bz = (float)k - vc.z * sdt;
    WTaps tb, tf;
    wtaps(t, bx, by, bz, tb);
    float3 vf = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int64_t r = tb.s[q];
        vf.x = vf.x + __ldg(vel + 3 * r) * tb.w[q];
        vf.y = vf.y + __ldg(vel + 3 * r + 1) * tb.w[q];
        vf.z = vf.z + __ldg(vel + 3 * r + 2) * tb.w[q];
    }
    wtaps(t, bx + vf.x * sdt, by + vf.y * sdt, bz + vf.z * sdt, tf);
    const float po = __ldg(d + s);
    float pf = 0.f, pb = 0.f;
    float3 gpf = make_float3(0.f, 0.f, 0.f), gpb = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float a = __ldg(d + tb.s[q]), b = __ldg(d + tf.s[q]);
        pf = __fmaf_rn(a, tb.w[q], pf);
        pb = __fmaf_rn(b, tf.w[q], pb);
        gpf.x += a * tb.gx[q], gpf.y += a * tb.gy[q], gpf.z += a * tb.gz[q];
        gpb.x += b * tf.gx[q], gpb.y += b * tf.gy[q], gpb.z += b * tf.gz[q];
    }
    const float corr = __fmaf_rn(0.5f, po - pb, pf);
    // The clamp set in the forward's order: centre, x-1, x+1, y-1, y+1, z-1, z+1, the forward sample.
    const int64_t ns[6] = {slot0(t, i - 1, j, k), slot0(t, i + 1, j, k), slot0(t, i, j - 1, k),
                           slot0(t, i, j + 1, k), slot0(t, i, j, k - 1), slot0(t, i, j, k + 1)};
    float mn = po, mx = po;
    int imn = -2, imx = -2;  // -2 centre, 0..5 a neighbour, 6 the forward sample
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float a = __ldg(d + ns[q]);
        if (a < mn) mn = a, imn = q;
        if (a > mx) mx = a, imx = q;
    }
    if (pf < mn) mn = pf, imn = 6;
    if (pf > mx) mx = pf, imx = 6;
    const int pick = corr > mx ? imx : corr < mn ? imn : -1;
    float g_po = 0.f, g_pf = 0.f, g_pb = 0.f;
    if (pick == -1) {
        g_pf = ob, g_po = 0.5f * ob, g_pb = -0.5f * ob;
    } else if (pick == -2) {
        g_po = ob;
    } else if (pick == 6) {
        g_pf = ob;
    } else {
        atomicAdd(d_bar + ns[pick], ob);
    }
    if (g_po != 0.f) atomicAdd(d_bar + s, g_po);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (g_pf != 0.f) atomicAdd(d_bar + tb.s[q], g_pf * tb.w[q]);
        if (g_pb != 0.f) atomicAdd(d_bar + tf.s[q], g_pb * tf.w[q]);
    }
    // Positions: pf at back, pb at fwd = back + vf(back) sdt, back = x - vc sdt.
    const float3 fb = make_float3(g_pb * gpb.x, g_pb * gpb.y, g_pb * gpb.z);
    float3 bb = make_float3(g_pf * gpf.x + fb.x, g_pf * gpf.y + fb.y, g_pf * gpf.z + fb.z);
    const float3 vfb = make_float3(fb.x * sdt, fb.y * sdt, fb.z * sdt);
    if (vfb.x != 0.f || vfb.y != 0.f || vfb.z != 0.f) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int64_t r = tb.s[q];
            atomicAdd(vel_bar + 3 * r, vfb.x * tb.w[q]);
            atomicAdd(vel_bar + 3 * r + 1, vfb.y * tb.w[q]);
            atomicAdd(vel_bar + 3 * r + 2, vfb.z * tb.w[q]);
            const float ux = __ldg(vel + 3 * r), uy = __ldg(vel + 3 * r + 1), uz = __ldg(vel + 3 * r + 2);
            const float dv = vfb.x * ux + vfb.y * uy + vfb.z * uz;
            bb.x += dv * tb.gx[q], bb.y += dv * tb.gy[q], bb.z += dv * tb.gz[q];
        }
    }
    if (bb.x != 0.f) atomicAdd(vel_bar + 3 * s, -sdt * bb.x);
    if (bb.y != 0.f) atomicAdd(vel_bar + 3 * s + 1, -sdt * bb.y);
    if (bb.z != 0.f) atomicAdd(vel_bar + 3 * s + 2, -sdt * bb.z);
}

// s1 = s + dt src (add_scalar_source, out of place; the forward's arithmetic).
__global__ void __launch_bounds__(kThreads) add_source_kernel(const float* __restrict__ in, const float* __restrict__ src,
                                                              float* __restrict__ out, float dt, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s < n) out[s] = src ? in[s] + dt * __ldg(src + s) : in[s];
}

struct PointwiseIn {
    const float* s1[kFields];  // the fields after the sources, before the burn (null: absent)
    const float* mid_bar[kFields];  // adjoints of the burned fields (what the advection read)
    float* in_bar[kFields];    // the step's input adjoints (+=)
};

// Transposes of the sources (identity), the burn and the buoyancy, per voxel. adv3_bar: the
// adjoint of the forced velocity before the projection; div_bar: of the divergence (the
// oxygen burn's expansion term).
template <int kModel>
__global__ void __launch_bounds__(kThreads) adj_burn_buoy_kernel(PointwiseIn P, const float* __restrict__ adv3_bar,
                                                                 const float* __restrict__ div_bar, float gain,
                                                                 float expansion, float rate, float heat, float ignition,
                                                                 float alpha, float dt, float ambient, float strength,
                                                                 int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (s >= n) return;
    auto val = [&](int f) { return P.s1[f] ? P.s1[f][s] : 0.f; };
    auto bar = [&](int f) { return P.mid_bar[f] ? P.mid_bar[f][s] : 0.f; };
    const float T1 = val(kT), F1 = val(kF), W = val(kW), FL = val(kFL);
    // The burn, recomputed, with its branches.
    float T2 = T1, dbF = 0.f, dbW = 0.f, dF = 1.f, dFLb = 0.f;
    bool burning = false, fl_keeps = true;
    if constexpr (kModel == HNS_COMBUSTION_RATE) {
        if (F1 > 0.0f && T1 >= ignition) {
            const float rdt = rate * dt, b = fminf(F1, rdt);
            burning = true;
            dbF = F1 < rdt ? 1.f : 0.f;
            T2 = T1 + b * heat;
        }
    } else if constexpr (kModel == HNS_COMBUSTION_OXYGEN) {
        float F = F1;
        if (F < 0.001f) F = 0.0f, dF = 0.f;
        const float oxy = 1.0f - F - W;
        if (oxy >= 0.0f) {
            burning = true;
            const float burn = fminf(oxy, F);
            if (oxy < F) dbF = -1.f, dbW = -1.f;
            else dbF = 1.f, dbW = 0.f;
            T2 = T1 + burn * gain;
            const float cand = fminf(1.0f, burn * 10.0f);
            fl_keeps = FL >= cand;
            dFLb = (!fl_keeps && burn * 10.0f < 1.0f) ? 10.f : 0.f;
        }
    }
    // Buoyancy: adv3.y = adv2.y + (b_T(T2) - alpha D1) dt.
    const float ay = adv3_bar[3 * s + 1] * dt;
    const float dbt = (T2 > ambient && (T2 - ambient) * strength > 0.0f) ? strength : 0.0f;
    const float T2b = bar(kT) + ay * dbt;
    const float D1b = bar(kD) - ay * alpha;
    float T1b = T2b, F1b = bar(kF), Wb = bar(kW), FLb = bar(kFL);
    if constexpr (kModel == HNS_COMBUSTION_RATE) {
        if (burning) {
            const float bb = -bar(kF) + T2b * heat;
            F1b = bar(kF) + bb * dbF;
        }
    } else if constexpr (kModel == HNS_COMBUSTION_OXYGEN) {
        if (burning) {
            const float bb = -bar(kF) + 2.0f * bar(kW) + gain * T2b + expansion * div_bar[s] + dFLb * bar(kFL);
            F1b = bar(kF) + bb * dbF;
            Wb = bar(kW) + bb * dbW;
            FLb = fl_keeps ? bar(kFL) : 0.f;
        }
        F1b *= dF;
    }
    // The sources are additive: the adjoints pass to the step's inputs unchanged.
    const float outb[kFields] = {D1b, T1b, F1b, Wb, FLb};
#pragma unroll
    for (int f = 0; f < kFields; ++f)
        if (P.in_bar[f]) P.in_bar[f][s] += outb[f];
}

float* sf(Context& c, const std::string& name, size_t count) { return c.scratch_f32("fire_adj_" + name, count); }

}  // namespace

// The projection of the adjoint: refined (exact) when solve is given, else `iterations` red-black
// iterations (omega as the step uses it).
struct FireAdjointSolve {
    int iterations = 0;
    float omega = 0.f;
    const hns_mixed_desc* refined = nullptr;
};

void adjoint_fire(Context& c, const hns_fire_f32& in, const hns_fire_sources_f32& src, const hns_fire_f32& out_bar,
                  const hns_fire_f32& in_bar, float dt, const hns_combustion_params& P, const hns_force_model& M,
                  const FireAdjointSolve& S) {
    const size_t n = (size_t)c.num_voxels();
    const int64_t nn = (int64_t)n;
    const float* sin[kFields] = {in.density, in.temperature, in.fuel, in.waste, in.flame};
    const float* sbar_out[kFields] = {out_bar.density, out_bar.temperature, out_bar.fuel, out_bar.waste, out_bar.flame};
    float* sbar_in[kFields] = {in_bar.density, in_bar.temperature, in_bar.fuel, in_bar.waste, in_bar.flame};
    const float* srcs[kFields] = {src.density, src.temperature, src.fuel, nullptr, nullptr};
    static const char* nm[kFields] = {"density", "temperature", "fuel", "waste", "flame"};

    // ---- the forward, recomputed ----
    float* adv = sf(c, "adv", 3 * n);
    float* adv2 = sf(c, "adv2", 3 * n);
    float* adv3 = sf(c, "adv3", 3 * n);
    float* div = sf(c, "div", n);
    FieldSet none{};
    launch_advect_fused(c, in.velocity, adv, none, dt);
    launch_confine_sources(c, adv, adv2, dt, P.vorticityScale, P.factorScale, src.velocity, P.gravity);
    float* s1[kFields] = {};
    float* s2[kFields] = {};
    for (int f = 0; f < kFields; ++f) {
        if (!sin[f]) continue;
        s1[f] = sf(c, std::string("s1_") + nm[f], n);
        s2[f] = sf(c, std::string("s2_") + nm[f], n);
        add_source_kernel<<<blocks_for(nn), kThreads, 0, c.stream>>>(sin[f], srcs[f], s1[f], dt, nn);
        HNS_LAUNCHED();
        HNS_CUDA(cudaMemcpyAsync(s2[f], s1[f], n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
    }
    launch_div_combust_buoy(c, adv2, adv3, div, s2[kF], s2[kW], s2[kT], s2[kFL],
                            M.density_buoyancy != 0.0f ? s2[kD] : nullptr, P, M, dt);
    float* velp = sf(c, "velp", 3 * n);
    double* p64 = nullptr;
    if (S.refined) {
        p64 = reinterpret_cast<double*>(sf(c, "p64", 2 * n));
        const float om = S.refined->omega > 0.f ? S.refined->omega : 1.9f;
        refine_solve<__half>(c, div, p64, S.refined->max_outer, S.refined->inner_iterations, om, S.refined->tolerance,
                             S.refined->flags);
        HNS_CUDA(cudaMemcpyAsync(velp, adv3, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
        launch_gradient_f64(c, velp, p64);
    } else {
        float* p = sf(c, "p", n);
        rbgs_solve(c, div, p, S.iterations, S.omega, HNS_SOLVE_ZERO_INIT);
        launch_subtract_gradient(c, adv3, p, velp);
    }

    // ---- reverse ----
    float* vb = sf(c, "vb", 3 * n);
    HNS_CUDA(cudaMemcpyAsync(vb, out_bar.velocity, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
    float* mid[kFields] = {};
    for (int f = 0; f < kFields; ++f) {
        if (!sin[f]) continue;
        mid[f] = sf(c, std::string("mid_") + nm[f], n);
        HNS_CUDA(cudaMemsetAsync(mid[f], 0, n * sizeof(float), c.stream));
        if (sbar_out[f]) {
            adj_advect_scalars_kernel<<<blocks_for(nn), kThreads, 0, c.stream>>>(c.topo.view, velp, s2[f], sbar_out[f],
                                                                                 mid[f], vb, dt * (1.0f / c.dx), nn);
            HNS_LAUNCHED();
        }
    }
    // The projection: vel' = adv3 - grad p, p = M div.
    float* pbar = sf(c, "pbar", n);
    float* dbar = sf(c, "dbar", n);
    HNS_CUDA(cudaMemsetAsync(pbar, 0, n * sizeof(float), c.stream));
    HNS_CUDA(cudaMemsetAsync(dbar, 0, n * sizeof(float), c.stream));
    launch_adj_gradient(c, vb, pbar);
    if (S.refined) {
        // div_bar = dx^2 L^-1 p_bar: the refined solve of p_bar as a divergence.
        const float om = S.refined->omega > 0.f ? S.refined->omega : 1.9f;
        refine_solve<__half>(c, pbar, p64, S.refined->max_outer, S.refined->inner_iterations, om, S.refined->tolerance,
                             S.refined->flags);
        convert_array(c, p64, HNS_DTYPE_F64, dbar, HNS_DTYPE_F32, nn);
    } else {
        adj_rbgs(c, pbar, dbar, S.iterations, S.omega);
    }
    // adv2_bar = adv3_bar (the buoyancy adds to adv2) + D^T div_bar.
    float* adv2b = sf(c, "adv2b", 3 * n);
    HNS_CUDA(cudaMemcpyAsync(adv2b, vb, 3 * n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
    launch_adj_divergence(c, dbar, adv2b);
    // Burn, buoyancy and sources, per voxel.
    PointwiseIn pin{};
    for (int f = 0; f < kFields; ++f) {
        pin.s1[f] = s1[f];
        pin.mid_bar[f] = mid[f];
        pin.in_bar[f] = sin[f] ? sbar_in[f] : nullptr;
    }
    const unsigned g = blocks_for(nn);
    if (M.combustion == HNS_COMBUSTION_OXYGEN)
        adj_burn_buoy_kernel<HNS_COMBUSTION_OXYGEN><<<g, kThreads, 0, c.stream>>>(
            pin, vb, dbar, P.temperatureRelease, P.expansionRate, M.burn_rate, M.heat_release, M.ignition_temp,
            M.density_buoyancy, dt, P.ambientTemp, P.buoyancyStrength, nn);
    else if (M.combustion == HNS_COMBUSTION_RATE)
        adj_burn_buoy_kernel<HNS_COMBUSTION_RATE><<<g, kThreads, 0, c.stream>>>(
            pin, vb, dbar, P.temperatureRelease, P.expansionRate, M.burn_rate, M.heat_release, M.ignition_temp,
            M.density_buoyancy, dt, P.ambientTemp, P.buoyancyStrength, nn);
    else
        adj_burn_buoy_kernel<HNS_COMBUSTION_NONE><<<g, kThreads, 0, c.stream>>>(
            pin, vb, dbar, P.temperatureRelease, P.expansionRate, M.burn_rate, M.heat_release, M.ignition_temp,
            M.density_buoyancy, dt, P.ambientTemp, P.buoyancyStrength, nn);
    HNS_LAUNCHED();
    // Confinement and the velocity's self-advection.
    float* advb = sf(c, "advb", 3 * n);
    HNS_CUDA(cudaMemsetAsync(advb, 0, 3 * n * sizeof(float), c.stream));
    launch_adj_confinement(c, adv, adv2b, advb, dt, P.vorticityScale, P.factorScale);
    launch_adj_advect_vec3(c, in.velocity, advb, in_bar.velocity, dt);
}

}  // namespace hns

using namespace hns;

namespace {

void check_fire_adjoint(const hns_fire_f32* out_bar, const hns_fire_f32* in_bar, const hns_combustion_params* params,
                        const hns_force_model& M) {
    if (!out_bar || !in_bar || !params) fail(HNS_ERR_INVALID_ARG, "null argument");
    if (!out_bar->velocity || !in_bar->velocity) fail(HNS_ERR_INVALID_ARG, "the velocity adjoints are required");
    if (params->substeps > 1) fail(HNS_ERR_UNSUPPORTED, "the fire adjoint takes one substep");
    if (params->disturbanceEnable > 0.0f) fail(HNS_ERR_UNSUPPORTED, "the fire adjoint takes no disturbance re-solve");
    check_force_model(M);
}

void check_fields_f32(const hns_fire_f32& in, const hns_fire_f32& out_bar, const hns_fire_f32& in_bar,
                      const hns_force_model& M) {
    const float* a[6] = {in.velocity, in.density, in.temperature, in.fuel, in.waste, in.flame};
    const float* b[6] = {in_bar.velocity, in_bar.density, in_bar.temperature, in_bar.fuel, in_bar.waste, in_bar.flame};
    for (int q = 0; q < 6; ++q)
        if ((a[q] == nullptr) != (b[q] == nullptr)) fail(HNS_ERR_INVALID_ARG, "each field needs its input adjoint");
    (void)out_bar;
    if (!in.temperature) fail(HNS_ERR_INVALID_ARG, "the step needs a temperature field");
    if (M.combustion != HNS_COMBUSTION_NONE && !in.fuel) fail(HNS_ERR_INVALID_ARG, "the burn needs a fuel field");
    if (M.combustion == HNS_COMBUSTION_OXYGEN && (!in.waste || !in.flame))
        fail(HNS_ERR_INVALID_ARG, "the oxygen burn needs waste and flame fields");
    if (M.density_buoyancy != 0.0f && !in.density) fail(HNS_ERR_INVALID_ARG, "the density buoyancy needs a density field");
}

}  // namespace

extern "C" {

HNS_API hns_status hns_adjoint_advance(hns_ctx* ctx, const hns_fire_f32* in, const hns_fire_sources_f32* sources,
                                       const hns_fire_f32* out_bar, const hns_fire_f32* in_bar, float dt, int iterations,
                                       const hns_combustion_params* params, const hns_force_model* model) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!in || !in->velocity) fail(HNS_ERR_INVALID_ARG, "null fields");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        const hns_force_model M = model ? *model : hns_force_model{};
        check_fire_adjoint(out_bar, in_bar, params, M);
        check_fields_f32(*in, *out_bar, *in_bar, M);
        DeviceGuard dg(c->device);
        FireAdjointSolve S;
        S.iterations = iterations;
        S.omega = 2.0f / (1.0f + sinf(3.14159f * c->dx));  // HNS_Advance's (src/Cuda/HNanoSolver.cu:365)
        adjoint_fire(*c, *in, sources ? *sources : hns_fire_sources_f32{}, *out_bar, *in_bar, dt, *params, M, S);
    });
}

HNS_API hns_status hns_adjoint_advance_mixed(hns_ctx* ctx, const hns_fire_fields* in, const hns_fire_sources* sources,
                                             const hns_fire_f32* out_bar, const hns_fire_f32* in_bar, float dt,
                                             const hns_combustion_params* params, const hns_force_model* model,
                                             const hns_mixed_desc* solve) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!in || !in->velocity || !solve) fail(HNS_ERR_INVALID_ARG, "null fields or solve description");
        if (solve->max_outer <= 0 || solve->max_outer > 1000 || solve->inner_iterations <= 0 || !(solve->tolerance > 0.0))
            fail(HNS_ERR_INVALID_ARG, "bad solve description");
        const hns_force_model M = model ? *model : hns_force_model{};
        check_fire_adjoint(out_bar, in_bar, params, M);
        DeviceGuard dg(c->device);
        const size_t n = (size_t)c->num_voxels();
        // The BF16/FP16 inputs as FP32: the step's arithmetic is FP32 on these values.
        const void* hin[6] = {in->velocity, in->density, in->temperature, in->fuel, in->waste, in->flame};
        static const char* nm[6] = {"velocity", "density", "temperature", "fuel", "waste", "flame"};
        float* f32[6] = {};
        for (int q = 0; q < 6; ++q) {
            if (!hin[q]) continue;
            if (((uintptr_t)hin[q]) & 1u) fail(HNS_ERR_INVALID_ARG, "BF16/FP16 arrays must be 2-byte aligned");
            const size_t cnt = q == 0 ? 3 * n : n;
            f32[q] = c->scratch_f32(std::string("fire_adjm_in_") + nm[q], cnt);
            convert_array(*c, hin[q], q == 0 ? HNS_DTYPE_BF16 : HNS_DTYPE_F16, f32[q], HNS_DTYPE_F32, (int64_t)cnt);
        }
        const hns_fire_f32 fin{f32[0], f32[1], f32[2], f32[3], f32[4], f32[5]};
        check_fields_f32(fin, *out_bar, *in_bar, M);
        hns_fire_sources_f32 fs{};
        if (sources) {
            const void* hs[4] = {sources->velocity, sources->temperature, sources->density, sources->fuel};
            const float** ps[4] = {&fs.velocity, &fs.temperature, &fs.density, &fs.fuel};
            static const char* sn[4] = {"velocity", "temperature", "density", "fuel"};
            for (int q = 0; q < 4; ++q) {
                if (!hs[q]) continue;
                const size_t cnt = q == 0 ? 3 * n : n;
                float* d = c->scratch_f32(std::string("fire_adjm_src_") + sn[q], cnt);
                convert_array(*c, hs[q], q == 0 ? HNS_DTYPE_BF16 : HNS_DTYPE_F16, d, HNS_DTYPE_F32, (int64_t)cnt);
                *ps[q] = d;
            }
        }
        FireAdjointSolve S;
        S.refined = solve;
        adjoint_fire(*c, fin, fs, *out_bar, *in_bar, dt, *params, M, S);
    });
}

}  // extern "C"
