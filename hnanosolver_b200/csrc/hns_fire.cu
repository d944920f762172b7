// The all-in-one step (HNS_Advance, src/Cuda/HNanoSolver.cu:223-456) on reduced-precision
// storage: BF16 velocity and FP16 scalars (density, temperature, fuel, waste, flame), FP32
// arithmetic, and the pressure solves as the FP64 iterative refinement of hns_step_mixed.
//
// Per substep:
//   advect_records / advect_mixed   velocity -> adv                     (advect_vector)
//   confine_mixed                   adv -> adv2, + velocity source,     (vorticityConfinement out
//                                   gravity                              of place, add_velocity_source,
//                                                                        add_gravity)
//   div_burn_buoy_mixed             adv2 -> div, adv3 (= out velocity);  (divergence, add_scalar_source,
//                                   scalars -> burned scalars            the force model's burn,
//                                                                        temperature_buoyancy [+ density])
//   refined solve                   div -> p (FP64)                      (redBlackGaussSeidelUpdate loop,
//   [divergence of adv3, refined solve]  disturbanceEnable > 0           to a tolerance)
//   gradient_mixed                  out velocity -= grad p, in place     (subtractPressureGradient)
//   pack_fire_records +             scalars -> out scalars along the     (advect_scalars)
//   advect_scalars_records          projected velocity
// The scalar sources are pointwise and independent of the velocity, so adding them in the
// divergence pass instead of the confinement pass (where HNS_Advance launches them) gives the
// same values, and the sourced value feeds the burn in FP32 without an FP16 rounding between.
// Each field is read and written once per pass at its storage width; the burned scalars go to
// solver-owned FP16 arrays only for the fields the pass changes.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "hns_confine.cuh"
#include "hns_internal.cuh"
#include "hns_stencil.cuh"
#include "hns_types.cuh"

namespace hns {
namespace {

using namespace dev;

constexpr int kThreads = 256;
using bf16 = __nv_bfloat16;

unsigned leaf_blocks(const Context& c) { return (unsigned)(c.topo.num_leaves * 2); }

// Nearest read of a reduced-precision vec3 field, 0 outside the domain.
__device__ __forceinline__ float3 near_b(const TopoView& t, const LeafNbhd& L, const bf16* __restrict__ d, int i, int j,
                                         int k) {
    const int64_t s = slot_of(t, L, i, j, k);
    return s < 0 ? make_float3(0.f, 0.f, 0.f) : vload(d, s);
}

// |curl u| at a voxel (computeVorticityMag, src/Cuda/Utils.cuh:226-243) on BF16 storage.
__device__ __forceinline__ float vort_mag_b(const TopoView& t, const LeafNbhd& L, const bf16* __restrict__ v, int i, int j,
                                            int k, float factor) {
    const float3 px = near_b(t, L, v, i + 1, j, k), mx = near_b(t, L, v, i - 1, j, k);
    const float3 py = near_b(t, L, v, i, j + 1, k), my = near_b(t, L, v, i, j - 1, k);
    const float3 pz = near_b(t, L, v, i, j, k + 1), mz = near_b(t, L, v, i, j, k - 1);
    const float ox = ((py.z - my.z) - (pz.y - mz.y)) * factor;
    const float oy = ((pz.x - mz.x) - (px.z - mx.z)) * factor;
    const float oz = ((px.y - mx.y) - (py.x - my.x)) * factor;
    return __fsqrt_rn(ox * ox + oy * oy + oz * oz);
}

// vorticityConfinement (src/Cuda/Kernel.cu:682-727) out of place, then the velocity source
// (add_velocity_source, Kernel.cu:739-745) and gravity (add_gravity, Kernel.cu:834-838), in
// the order HNS_Advance launches them (src/Cuda/HNanoSolver.cu:279-318), on BF16 storage with
// the FP32 step's operation order.
__global__ void __launch_bounds__(kThreads) confine_mixed_kernel(TopoView t, const bf16* __restrict__ vel,
                                                                  bf16* __restrict__ out, float dt, float inv_dx,
                                                                  float scale, int fs, const bf16* __restrict__ src_v3,
                                                                  float gravity) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float factor = 0.5f * inv_dx;
    const float3 px = near_b(t, L, vel, i + 1, j, k), mx = near_b(t, L, vel, i - 1, j, k);
    const float3 py = near_b(t, L, vel, i, j + 1, k), my = near_b(t, L, vel, i, j - 1, k);
    const float3 pz = near_b(t, L, vel, i, j, k + 1), mz = near_b(t, L, vel, i, j, k - 1);
    const float ox = ((py.z - my.z) - (pz.y - mz.y)) * factor;
    const float oy = ((pz.x - mz.x) - (px.z - mx.z)) * factor;
    const float oz = ((px.y - mx.y) - (py.x - my.x)) * factor;
    const float mpx = vort_mag_b(t, L, vel, i + fs, j, k, factor), mmx = vort_mag_b(t, L, vel, i - fs, j, k, factor);
    const float mpy = vort_mag_b(t, L, vel, i, j + fs, k, factor), mmy = vort_mag_b(t, L, vel, i, j - fs, k, factor);
    const float mpz = vort_mag_b(t, L, vel, i, j, k + fs, factor), mmz = vort_mag_b(t, L, vel, i, j, k - fs, factor);
    const float gx = (mpx - mmx) * 0.5f * inv_dx;
    const float gy = (mpy - mmy) * 0.5f * inv_dx;
    const float gz = (mpz - mmz) * 0.5f * inv_dx;
    const float glen = sqrtf(gx * gx + gy * gy + gz * gz) + 1e-5f;
    const float nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const float3 u = vload(vel, s);
    const float fx = scale * (ny * oz - nz * oy), fy = scale * (nz * ox - nx * oz), fz = scale * (nx * oy - ny * ox);
    float3 r = make_float3(u.x + fx * dt, u.y + fy * dt, u.z + fz * dt);
    if (src_v3 != nullptr) {
        const float3 a = vload(src_v3, s);
        r.x += a.x * dt;
        r.y += a.y * dt;
        r.z += a.z * dt;
    }
    if (gravity != 0.0f) r.y -= gravity * dt;
    vstore(out, s, r);
}

// confine_mixed_kernel on a shared-memory leaf tile (hns_confine.cuh), for |fs| <= 1: one CTA
// per leaf, the same values.
__global__ void __launch_bounds__(kThreads) confine_tile_mixed_kernel(TopoView t, const bf16* __restrict__ vel,
                                                                       bf16* __restrict__ out, float dt, float inv_dx,
                                                                       float scale, int fs, const bf16* __restrict__ src_v3,
                                                                       float gravity) {
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
            const float3 a = vload(src_v3, s);
            r.x += a.x * dt;
            r.y += a.y * dt;
            r.z += a.z * dt;
        }
        if (gravity != 0.0f) r.y -= gravity * dt;
        vstore(out, s, r);
    }
}

// The scalar fields of one pass (FP16; null: absent) and the burned outputs (null: the pass
// leaves that field unchanged and writes nothing).
struct FireScalars {
    const __half* temp_in;
    const __half* fuel_in;
    const __half* waste_in;
    const __half* flame_in;
    const __half* dens_in;
    const __half* src_temp;
    const __half* src_fuel;
    const __half* src_dens;
    __half* temp_out;
    __half* fuel_out;
    __half* waste_out;
    __half* flame_out;
    __half* dens_out;
};

struct BurnParams {
    float gain, expansion;       // combustion_oxygen: temperatureRelease, expansionRate
    float rate, heat, ignition;  // combustion: burn rate, heat release, ignition temperature
    float alpha;                 // density buoyancy; 0: the reference's temperature_buoyancy
};

__device__ __forceinline__ float opt_load(const __half* p, int64_t s) { return p != nullptr ? sload(p, s) : 0.0f; }

// divergence (Kernel.cu:432-453) of the forced velocity; the scalar sources (add_scalar_source,
// Kernel.cu:732-737: temperature, density, fuel); the force model's burn (combustion_oxygen,
// Kernel.cu:641-677, with the expansion added to the divergence; combustion, Kernel.cu:568-588;
// or none); then temperature_buoyancy (Kernel.cu:546-563) from the burned temperature, with the
// density term when alpha != 0, into vel_out (neighbouring threads still read vel).
template <int kModel>
__global__ void __launch_bounds__(kThreads) div_burn_buoy_mixed_kernel(TopoView t, const bf16* __restrict__ vel,
                                                                        bf16* __restrict__ vel_out, float* __restrict__ div,
                                                                        float inv_dx, FireScalars S, BurnParams B, float dt,
                                                                        float ambient, float strength) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const int64_t s = (v.leaf << 9) + v.n;
    const float3 c = vload(vel, s);
    const float xp = (c.x + near_b(t, L, vel, i + 1, j, k).x) * 0.5f;
    const float xm = (c.x + near_b(t, L, vel, i - 1, j, k).x) * 0.5f;
    const float yp = (c.y + near_b(t, L, vel, i, j + 1, k).y) * 0.5f;
    const float ym = (c.y + near_b(t, L, vel, i, j - 1, k).y) * 0.5f;
    const float zp = (c.z + near_b(t, L, vel, i, j, k + 1).z) * 0.5f;
    const float zm = (c.z + near_b(t, L, vel, i, j, k - 1).z) * 0.5f;
    float dv = (xp - xm + yp - ym + zp - zm) * inv_dx;

    float T = opt_load(S.temp_in, s);
    if (S.src_temp != nullptr) T += dt * sload(S.src_temp, s);
    float D = opt_load(S.dens_in, s);
    if (S.src_dens != nullptr) D += dt * sload(S.src_dens, s);
    float F = opt_load(S.fuel_in, s);
    if (S.src_fuel != nullptr) F += dt * sload(S.src_fuel, s);
    if constexpr (kModel == HNS_COMBUSTION_OXYGEN) {
        float W = sload(S.waste_in, s), FL = sload(S.flame_in, s);
        if (F < 0.001f) F = 0.0f;
        const float oxy = 1.0f - F - W;
        if (oxy >= 0.0f) {
            const float burn = fminf(oxy, F);
            F = F - burn;
            W = W + burn * 2.0f;
            T = T + burn * B.gain;
            dv += burn * B.expansion;
            FL = fmaxf(FL, fminf(1.0f, burn * 10.0f));
        }
        sstore(S.waste_out, s, W);
        sstore(S.flame_out, s, FL);
    } else if constexpr (kModel == HNS_COMBUSTION_RATE) {
        if (F > 0.0f && T >= B.ignition) {
            const float burned = fminf(F, B.rate * dt);
            F = F - burned;
            T = T + burned * B.heat;
        }
    }
    div[s] = dv;
    if (S.temp_out != nullptr) sstore(S.temp_out, s, T);
    if (S.fuel_out != nullptr) sstore(S.fuel_out, s, F);
    if (S.dens_out != nullptr) sstore(S.dens_out, s, D);
    float3 r = c;
    if (B.alpha != 0.0f) {
        const float bt = T > ambient ? fmaxf(0.0f, (T - ambient) * strength) : 0.0f;
        r.y = c.y + (bt - B.alpha * D) * dt;
    } else if (T > ambient) {
        r.y = c.y + fmaxf(0.0f, (T - ambient) * strength) * dt;
    }
    vstore(vel_out, s, r);
}

constexpr int kFireFields = 5;  // density, temperature, fuel, waste, flame

struct HalfFields {
    const __half* in[kFireFields];
    __half* out[kFireFields];
    int count;
};

// Voxel records for the scalar advection: the BF16 velocity and up to five FP16 scalars in 16
// bytes (u | v << 16, w | s0 << 16, s1 | s2 << 16, s3 | s4 << 16; absent scalars 0), so that each
// of the 2 x 8 trace taps and 6 clamp neighbours is one load instead of one per field.
__global__ void __launch_bounds__(kThreads) pack_fire_records_kernel(const bf16* __restrict__ vel, HalfFields f,
                                                                      uint4* __restrict__ rec, int64_t n) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        const unsigned short* v = reinterpret_cast<const unsigned short*>(vel) + 3 * s;
        uint32_t h[kFireFields] = {0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for (int q = 0; q < kFireFields; ++q)
            if (q < f.count) h[q] = __half_as_ushort(__ldg(f.in[q] + s));
        rec[s] = make_uint4((uint32_t)__ldg(v) | ((uint32_t)__ldg(v + 1) << 16), (uint32_t)__ldg(v + 2) | (h[0] << 16),
                            h[1] | (h[2] << 16), h[3] | (h[4] << 16));
    }
}

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }
__device__ __forceinline__ float hf(uint32_t w, int hi) {
    return __half2float(__ushort_as_half((unsigned short)(hi ? (w >> 16) : (w & 0xFFFFu))));
}
// Scalar q of a record (word 1 high half, then words 2 and 3).
__device__ __forceinline__ float rec_s(const uint4& r, int q) {
    return q == 0 ? hf(r.y, 1) : q == 1 ? hf(r.z, 0) : q == 2 ? hf(r.z, 1) : q == 3 ? hf(r.w, 0) : hf(r.w, 1);
}

// HNS_Advance's multi-field advection (advect_scalars, src/Cuda/Kernel.cu:163-289) on FP16
// fields along a BF16 velocity, from voxel records: the back-trace uses the voxel's own
// velocity, the taps' weight-sum trilinear (setupInterpolation, Kernel.cu:204-233) reads slot 0
// outside the domain, and the MacCormack correction is clamped to the centre, its six face
// neighbours and the forward sample; the FP32 step's operations in its order, one 16-byte load
// per tap for the velocity and every field.
// I: the slot type, int32_t where the grid has fewer than 2^22 leaves (32-bit addressing).
template <int kCount, typename I>
__global__ void __launch_bounds__(kThreads) advect_scalars_records_kernel(TopoView t, const uint4* __restrict__ rec,
                                                                           HalfFields f, float sdt) {
    __shared__ LeafNbhd L;
    const VoxelIdx v = voxel_of_block();
    load_nbhd(L, t, v.leaf);
    __syncthreads();
    const int i = (L.lx << 3) + (v.n >> 6), j = (L.ly << 3) + ((v.n >> 3) & 7), k = (L.lz << 3) + (v.n & 7);
    const I s = (I(v.leaf) << 9) + I(v.n);
    const uint4 o = __ldg(rec + s);
    const float bx = (float)i - bf_lo(o.x) * sdt, by = (float)j - bf_hi(o.x) * sdt, bz = (float)k - bf_lo(o.y) * sdt;
    I bi[8], fi[8], ni[6];
    float bw[8], fw[8];
    interp_setup_fast<I>(t, L, bx, by, bz, bi, bw);
    float3 vf = make_float3(0.f, 0.f, 0.f);
    float pf[kCount], pb[kCount];
#pragma unroll
    for (int c = 0; c < kCount; ++c) pf[c] = 0.f, pb[c] = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint4 a = __ldg(rec + bi[q]);
        vf.x = vf.x + bf_lo(a.x) * bw[q];
        vf.y = vf.y + bf_hi(a.x) * bw[q];
        vf.z = vf.z + bf_lo(a.y) * bw[q];
#pragma unroll
        for (int c = 0; c < kCount; ++c) pf[c] = __fmaf_rn(rec_s(a, c), bw[q], pf[c]);
    }
    interp_setup_fast<I>(t, L, bx + vf.x * sdt, by + vf.y * sdt, bz + vf.z * sdt, fi, fw);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint4 a = __ldg(rec + fi[q]);
#pragma unroll
        for (int c = 0; c < kCount; ++c) pb[c] = __fmaf_rn(rec_s(a, c), fw[q], pb[c]);
    }
    face_slots(L, s, v.n, ni);  // x-1, x+1, y-1, y+1, z-1, z+1
#pragma unroll
    for (int q = 0; q < 6; ++q) ni[q] = ni[q] < 0 ? I(0) : ni[q];  // outside the domain: slot 0
    float mn[kCount], mx[kCount], po[kCount];
#pragma unroll
    for (int c = 0; c < kCount; ++c) po[c] = rec_s(o, c), mn[c] = po[c], mx[c] = po[c];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const uint4 a = __ldg(rec + ni[q]);
#pragma unroll
        for (int c = 0; c < kCount; ++c) {
            const float x = rec_s(a, c);
            mn[c] = fminf(mn[c], x);
            mx[c] = fmaxf(mx[c], x);
        }
    }
#pragma unroll
    for (int c = 0; c < kCount; ++c) {
        const float corr = __fmaf_rn(0.5f, po[c] - pb[c], pf[c]);
        sstore(f.out[c], (int64_t)s, fmaxf(fminf(mn[c], pf[c]), fminf(corr, fmaxf(mx[c], pf[c]))));
    }
}

template <typename I>
void launch_advect_scalars_records(const Context& c, const uint4* rec, const HalfFields& f, float sdt) {
    const dim3 g = leaf_blocks(c);
    switch (f.count) {
        case 1: advect_scalars_records_kernel<1, I><<<g, kThreads, 0, c.stream>>>(c.topo.view, rec, f, sdt); break;
        case 2: advect_scalars_records_kernel<2, I><<<g, kThreads, 0, c.stream>>>(c.topo.view, rec, f, sdt); break;
        case 3: advect_scalars_records_kernel<3, I><<<g, kThreads, 0, c.stream>>>(c.topo.view, rec, f, sdt); break;
        case 4: advect_scalars_records_kernel<4, I><<<g, kThreads, 0, c.stream>>>(c.topo.view, rec, f, sdt); break;
        default: advect_scalars_records_kernel<5, I><<<g, kThreads, 0, c.stream>>>(c.topo.view, rec, f, sdt); break;
    }
    HNS_LAUNCHED();
}

// One substep's arrays: BF16 velocity and the five FP16 scalars (null: absent).
struct FireState {
    bf16* vel;
    __half* s[kFireFields];  // density, temperature, fuel, waste, flame
};

FireState state_of(const hns_fire_fields& f) {
    return FireState{static_cast<bf16*>(f.velocity),
                     {static_cast<__half*>(f.density), static_cast<__half*>(f.temperature), static_cast<__half*>(f.fuel),
                      static_cast<__half*>(f.waste), static_cast<__half*>(f.flame)}};
}

__half* half_scratch(Context& c, const std::string& name, size_t n) {
    return reinterpret_cast<__half*>(c.scratch_f32(name, (n + 1) / 2));
}

enum { kDensity = 0, kTemperature = 1, kFuel = 2, kWaste = 3, kFlame = 4 };

}  // namespace

// One HNS_Advance call on reduced-precision arrays; the result of the last refined solve is
// returned (its checks for hns_last_refine).
RefinePlan run_advance_mixed(Context& c, const hns_fire_fields& in, const hns_fire_fields& out, const hns_fire_sources& src,
                             float dt, const hns_combustion_params& P, const hns_force_model& M, const hns_mixed_desc& d) {
    const size_t n = (size_t)c.num_voxels();
    const float inv_dx = 1.0f / c.dx;
    const int subs = std::max(1, P.substeps);
    const float dt_sub = dt / (float)subs;
    const float omega = d.omega > 0.f ? d.omega : 1.9f;
    bf16* adv = reinterpret_cast<bf16*>(c.scratch_f32("fire_adv", (3 * n + 1) / 2));
    bf16* adv2 = reinterpret_cast<bf16*>(c.scratch_f32("fire_adv2", (3 * n + 1) / 2));
    float* div = c.scratch_f32("project_div", n);
    double* p = reinterpret_cast<double*>(c.scratch_f32("refine_p", 2 * n));
    const FireState fin = state_of(in), fout = state_of(out);
    const BurnParams B{P.temperatureRelease, P.expansionRate, M.burn_rate, M.heat_release, M.ignition_temp,
                       M.density_buoyancy};
    RefinePlan plan;
    FireState cur = fin;
    for (int sub = 0; sub < subs; ++sub) {
        // Intermediate substeps write solver-owned arrays; the last writes the caller's.
        FireState nxt = fout;
        if (sub + 1 < subs) {
            const std::string tag = "fire_sub" + std::to_string(sub & 1) + "_";
            nxt.vel = reinterpret_cast<bf16*>(c.scratch_f32(tag + "vel", (3 * n + 1) / 2));
            for (int q = 0; q < kFireFields; ++q)
                nxt.s[q] = fin.s[q] ? half_scratch(c, tag + std::to_string(q), n) : nullptr;
        }
        c.phase_begin(HNS_PHASE_ADVECT);
        launch_advect_mixed(c, cur.vel, adv, nullptr, nullptr, 0, dt_sub);
        c.phase_end();

        c.phase_begin(HNS_PHASE_FORCES);
        const int fs = (int)P.factorScale;
        if (fs >= -1 && fs <= 1)
            confine_tile_mixed_kernel<<<(unsigned)c.topo.num_leaves, kThreads, 0, c.stream>>>(
                c.topo.view, adv, adv2, dt_sub, inv_dx, P.vorticityScale, fs, static_cast<const bf16*>(src.velocity),
                P.gravity);
        else
            confine_mixed_kernel<<<leaf_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, adv, adv2, dt_sub, inv_dx, P.vorticityScale, fs, static_cast<const bf16*>(src.velocity),
                P.gravity);
        HNS_LAUNCHED();
        // The burned scalars: the fields this pass changes go to solver-owned arrays, which the
        // scalar advection then reads; the others are advected from the substep's input.
        FireScalars S{};
        S.dens_in = cur.s[kDensity];
        S.temp_in = cur.s[kTemperature];
        S.fuel_in = cur.s[kFuel];
        S.waste_in = cur.s[kWaste];
        S.flame_in = cur.s[kFlame];
        S.src_temp = static_cast<const __half*>(src.temperature);
        S.src_fuel = cur.s[kFuel] ? static_cast<const __half*>(src.fuel) : nullptr;
        S.src_dens = cur.s[kDensity] ? static_cast<const __half*>(src.density) : nullptr;
        const __half* adv_in[kFireFields] = {cur.s[0], cur.s[1], cur.s[2], cur.s[3], cur.s[4]};
        S.temp_out = half_scratch(c, "fire_burn_temperature", n);
        adv_in[kTemperature] = S.temp_out;
        if (cur.s[kFuel] && (M.combustion != HNS_COMBUSTION_NONE || S.src_fuel)) {
            S.fuel_out = half_scratch(c, "fire_burn_fuel", n);
            adv_in[kFuel] = S.fuel_out;
        }
        if (S.src_dens) {
            S.dens_out = half_scratch(c, "fire_burn_density", n);
            adv_in[kDensity] = S.dens_out;
        }
        if (M.combustion == HNS_COMBUSTION_OXYGEN) {
            S.waste_out = half_scratch(c, "fire_burn_waste", n);
            S.flame_out = half_scratch(c, "fire_burn_flame", n);
            adv_in[kWaste] = S.waste_out;
            adv_in[kFlame] = S.flame_out;
        }
        if (M.combustion == HNS_COMBUSTION_OXYGEN)
            div_burn_buoy_mixed_kernel<HNS_COMBUSTION_OXYGEN><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, adv2, nxt.vel, div, inv_dx, S, B, dt_sub, P.ambientTemp, P.buoyancyStrength);
        else if (M.combustion == HNS_COMBUSTION_RATE)
            div_burn_buoy_mixed_kernel<HNS_COMBUSTION_RATE><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, adv2, nxt.vel, div, inv_dx, S, B, dt_sub, P.ambientTemp, P.buoyancyStrength);
        else
            div_burn_buoy_mixed_kernel<HNS_COMBUSTION_NONE><<<leaf_blocks(c), kThreads, 0, c.stream>>>(
                c.topo.view, adv2, nxt.vel, div, inv_dx, S, B, dt_sub, P.ambientTemp, P.buoyancyStrength);
        HNS_LAUNCHED();
        c.phase_end();

        c.phase_begin(HNS_PHASE_SOLVE);
        plan = refine_solve<__half>(c, div, p, d.max_outer, d.inner_iterations, omega, d.tolerance, d.flags);
        if (P.disturbanceEnable > 0.0f) {
            // The reference's disturbance branch: the divergence again, without the expansion,
            // solved from p = 0 (src/Cuda/HNanoSolver.cu:377-403).
            launch_divergence_mixed(c, nxt.vel, div);
            plan = refine_solve<__half>(c, div, p, d.max_outer, d.inner_iterations, omega, d.tolerance, d.flags);
        }
        c.phase_end();
        c.last_refine = plan;
        c.phase_begin(HNS_PHASE_GRADIENT);
        launch_gradient_mixed(c, nxt.vel, p);
        c.phase_end();

        c.phase_begin(HNS_PHASE_ADVECT);
        HalfFields f{};
        for (int q = 0; q < kFireFields; ++q)
            if (cur.s[q]) {
                f.in[f.count] = adv_in[q];
                f.out[f.count] = nxt.s[q];
                ++f.count;
            }
        if (f.count > 0) {
            // Voxel records of the projected velocity and the fields, then one load per tap.
            uint4* rec = reinterpret_cast<uint4*>(c.scratch_f32("fire_records", 4 * n));
            const unsigned pg = (unsigned)std::min<int64_t>((int64_t)(n + kThreads - 1) / kThreads,
                                                            (int64_t)c.sm_count() * 8);
            pack_fire_records_kernel<<<pg, kThreads, 0, c.stream>>>(nxt.vel, f, rec, (int64_t)n);
            HNS_LAUNCHED();
            const float sdt = dt_sub * inv_dx;
            if (c.topo.num_leaves < (int64_t(1) << 22))
                launch_advect_scalars_records<int32_t>(c, rec, f, sdt);
            else
                launch_advect_scalars_records<int64_t>(c, rec, f, sdt);
        }
        c.phase_end();
        cur = nxt;
    }
    return plan;
}

}  // namespace hns

using namespace hns;

namespace {

void check_fire_fields(const hns_fire_fields* in, const hns_fire_fields* out, const hns_force_model& M) {
    if (!in || !out) fail(HNS_ERR_INVALID_ARG, "null field set");
    if (!in->velocity || !out->velocity || in->velocity == out->velocity)
        fail(HNS_ERR_INVALID_ARG, "bad velocity arrays (both needed, distinct)");
    const void* const a[6] = {in->velocity, in->density, in->temperature, in->fuel, in->waste, in->flame};
    const void* const b[6] = {out->velocity, out->density, out->temperature, out->fuel, out->waste, out->flame};
    static const char* names[6] = {"velocity", "density", "temperature", "fuel", "waste", "flame"};
    for (int q = 0; q < 6; ++q) {
        if ((a[q] == nullptr) != (b[q] == nullptr))
            fail(HNS_ERR_INVALID_ARG, std::string("field '") + names[q] + "' given on one side only");
        if (a[q] && a[q] == b[q]) fail(HNS_ERR_INVALID_ARG, std::string("field '") + names[q] + "' in and out alias");
        if ((((uintptr_t)a[q]) & 1u) || (((uintptr_t)b[q]) & 1u))
            fail(HNS_ERR_INVALID_ARG, std::string("field '") + names[q] + "' must be 2-byte aligned");
    }
    if (!in->temperature) fail(HNS_ERR_INVALID_ARG, "the step needs a temperature field");
    if (M.combustion != HNS_COMBUSTION_NONE && !in->fuel) fail(HNS_ERR_INVALID_ARG, "the burn needs a fuel field");
    if (M.combustion == HNS_COMBUSTION_OXYGEN && (!in->waste || !in->flame))
        fail(HNS_ERR_INVALID_ARG, "the oxygen burn needs waste and flame fields");
    if (M.density_buoyancy != 0.0f && !in->density) fail(HNS_ERR_INVALID_ARG, "the density buoyancy needs a density field");
}

}  // namespace

extern "C" {

HNS_API hns_status hns_advance_mixed(hns_ctx* ctx, const hns_fire_fields* in, const hns_fire_fields* out,
                                     const hns_fire_sources* sources, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model, const hns_mixed_desc* solve, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        if (!params || !solve) fail(HNS_ERR_INVALID_ARG, "null params or solve description");
        if (solve->max_outer <= 0 || solve->max_outer > 1000) fail(HNS_ERR_INVALID_ARG, "max_outer must be in [1, 1000]");
        if (solve->inner_iterations <= 0) fail(HNS_ERR_INVALID_ARG, "inner_iterations must be positive");
        if (!(solve->tolerance > 0.0) || !std::isfinite(solve->tolerance)) fail(HNS_ERR_INVALID_ARG, "tolerance must be positive");
        if (!std::isfinite(dt)) fail(HNS_ERR_INVALID_ARG, "bad dt");
        const hns_force_model M = model ? *model : hns_force_model{};
        check_force_model(M);
        check_fire_fields(in, out, M);
        const hns_fire_sources S = sources ? *sources : hns_fire_sources{};
        const void* const sp[4] = {S.velocity, S.temperature, S.density, S.fuel};
        for (const void* q : sp)
            if (((uintptr_t)q) & 1u) fail(HNS_ERR_INVALID_ARG, "source arrays must be 2-byte aligned");
        DeviceGuard dg(c->device);
        hns_mixed_desc d = *solve;
        d.dt = dt;
        const RefinePlan plan = run_advance_mixed(*c, *in, *out, S, dt, *params, M, d);
        if (info) {
            int outer = 0;
            double res = 0.0;
            refine_result(*c, plan, &outer, &res);
            info->iterations = outer * plan.inner;
            info->residual = res;
            info->initial_residual = 1.0;
            if (res > solve->tolerance)
                st = record_error(HNS_ERR_NOT_CONVERGED, "refined solve stopped after " + std::to_string(outer) +
                                                             " outer iterations with residual " + std::to_string(res));
        }
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_advance_mixed_host(hns_ctx* ctx, const hns_fire_f32* fields, const hns_fire_sources_f32* sources,
                                          float dt, const hns_combustion_params* params, const hns_force_model* model,
                                          const hns_mixed_desc* solve, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        if (!fields || !fields->velocity) fail(HNS_ERR_INVALID_ARG, "null host fields");
        DeviceGuard dg(c->device);
        const size_t n = (size_t)c->num_voxels();
        float* host[6] = {fields->velocity, fields->density, fields->temperature, fields->fuel, fields->waste, fields->flame};
        static const char* names[6] = {"velocity", "density", "temperature", "fuel", "waste", "flame"};
        float* stage = c->scratch_f32("fire_host_stage", 3 * n);
        hns_fire_fields in{}, out{};
        void** pin[6] = {&in.velocity, &in.density, &in.temperature, &in.fuel, &in.waste, &in.flame};
        void** pout[6] = {&out.velocity, &out.density, &out.temperature, &out.fuel, &out.waste, &out.flame};
        // Upload each host field in FP32 and convert it to its storage type (BF16 velocity,
        // FP16 scalars) in solver-owned arrays.
        for (int q = 0; q < 6; ++q) {
            if (!host[q]) continue;
            const size_t cnt = q == 0 ? 3 * n : n;
            const int dt_store = q == 0 ? HNS_DTYPE_BF16 : HNS_DTYPE_F16;
            *pin[q] = c->scratch_f32(std::string("fire_host_in_") + names[q], (cnt + 1) / 2);
            *pout[q] = c->scratch_f32(std::string("fire_host_out_") + names[q], (cnt + 1) / 2);
            HNS_CUDA(cudaMemcpyAsync(stage, host[q], cnt * sizeof(float), cudaMemcpyHostToDevice, c->stream));
            convert_array(*c, stage, HNS_DTYPE_F32, *pin[q], dt_store, (int64_t)cnt);
        }
        hns_fire_sources src{};
        if (sources) {
            const float* hs[4] = {sources->velocity, sources->temperature, sources->density, sources->fuel};
            const void** ps[4] = {&src.velocity, &src.temperature, &src.density, &src.fuel};
            static const char* sn[4] = {"velocity", "temperature", "density", "fuel"};
            for (int q = 0; q < 4; ++q) {
                if (!hs[q]) continue;
                const size_t cnt = q == 0 ? 3 * n : n;
                void* dst = c->scratch_f32(std::string("fire_host_src_") + sn[q], (cnt + 1) / 2);
                HNS_CUDA(cudaMemcpyAsync(stage, hs[q], cnt * sizeof(float), cudaMemcpyHostToDevice, c->stream));
                convert_array(*c, stage, HNS_DTYPE_F32, dst, q == 0 ? HNS_DTYPE_BF16 : HNS_DTYPE_F16, (int64_t)cnt);
                *ps[q] = dst;
            }
        }
        st = hns_advance_mixed(ctx, &in, &out, &src, dt, params, model, solve, info);
        if (st != HNS_OK && st != HNS_ERR_NOT_CONVERGED) fail(st, hns_last_error());
        // Convert back to FP32 and download in place.
        for (int q = 0; q < 6; ++q) {
            if (!host[q]) continue;
            const size_t cnt = q == 0 ? 3 * n : n;
            convert_array(*c, *pout[q], q == 0 ? HNS_DTYPE_BF16 : HNS_DTYPE_F16, stage, HNS_DTYPE_F32, (int64_t)cnt);
            HNS_CUDA(cudaMemcpyAsync(host[q], stage, cnt * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        }
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        if (st == HNS_ERR_NOT_CONVERGED) fail(st, "refined solve above the tolerance");
    });
    return g != HNS_OK ? g : st;
}

}  // extern "C"
