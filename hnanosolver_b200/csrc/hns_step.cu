// Pressure solve with device-side convergence checks, and the plain step of the SOP
// operator chain (HNanoAdvect + HNanoAdvectVelocity + HNanoProjectNonDivergent).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "hns_internal.cuh"

namespace hns {

// The FP32 colour-split workspace: the right-hand side and e (with the zero leaf after the last
// leaf) in the split layout, and the face table (shared with the FP16 inner solve's).
struct Split32 {
    float* rhs;
    float* e;
    int* nb8;
};

Split32 split32_workspace(Context& c) {
    Split32 w;
    w.rhs = c.scratch_f32("split32_rhs", (size_t)c.num_voxels());
    w.e = static_cast<float*>(c.split_e("split32_e", sizeof(float), 1));
    w.nb8 = c.split_faces();
    return w;
}

// `K` red-black iterations of the FP32 solve on colour-split leaves, result in p (slot order):
// the divergence and (unless HNS_SOLVE_ZERO_INIT) p are converted in, the half-sweeps run in place,
// and e is converted out. With a plan, the residual of the iterate check c reads is evaluated
// before iteration (c + 1) E - 1 into its slot and every later half-sweep tests the latest slot,
// the schedule of the staged kernel (rbgs_solve_checked), so both give the same iterates.
void split32_solve(Context& c, const float* div, float* p, int K, float omega, unsigned flags, const SolvePlan* plan) {
    const Split32 w = split32_workspace(c);
    const float dx2 = c.dx * c.dx;
    convert_split_f32(c, div, w.rhs, true);
    const bool zero = (flags & HNS_SOLVE_ZERO_INIT) != 0;
    if (!zero) convert_split_f32(c, p, w.e, true);
    const double tol2 = plan ? plan->tol * plan->tol : 0.0;
    if (c.split_solve == HNS_SPLIT_PERSISTENT) {
        // Persistent launches over the runs of iterations that share a check slot and have no
        // residual evaluation inside: [cE, (c+1)E - 1) and the single iteration (c+1)E - 1.
        for (int it = 0; it < K;) {
            const double* chk = nullptr;
            int end = K;
            if (plan) {
                const int E = plan->check_every;
                const int last_check = it / E - 1;
                chk = last_check >= 0 ? plan->slots + 2 * last_check : nullptr;
                if ((it + 1) % E == 0) {
                    launch_split_residual_f32(c, w.nb8, w.rhs, w.e, (double)dx2, chk, tol2,
                                              plan->slots + 2 * ((it + 1) / E - 1));
                    end = it + 1;
                } else {
                    end = std::min(K, (it / E + 1) * E - 1);
                }
            }
            launch_rbgs_split_solve_f32(c, w.nb8, w.rhs, w.e, 2 * (end - it), zero && it == 0, omega, dx2, chk, tol2);
            it = end;
        }
        convert_split_f32(c, w.e, p, false);
        return;
    }
    bool after_half = false;  // the preceding kernel on the stream is a half-sweep
    for (int it = 0; it < K; ++it) {
        const double* chk = nullptr;
        if (plan) {
            const int E = plan->check_every;
            const int last_check = it / E - 1;
            chk = last_check >= 0 ? plan->slots + 2 * last_check : nullptr;
            if ((it + 1) % E == 0) {
                launch_split_residual_f32(c, w.nb8, w.rhs, w.e, (double)dx2, chk, tol2, plan->slots + 2 * ((it + 1) / E - 1));
                after_half = false;
            }
        }
        launch_rbgs_split_half_f32(c, w.nb8, w.rhs, w.e, 0, zero && it == 0, omega, dx2, chk, tol2, false, after_half);
        launch_rbgs_split_half_f32(c, w.nb8, w.rhs, w.e, 1, false, omega, dx2, chk, tol2, false, true);
        after_half = true;
    }
    convert_split_f32(c, w.e, p, false);
}

bool use_split32(const Context& c, unsigned flags, const float* div, const float* p) {
    // The layout conversions move 16-byte vectors of div and p.
    auto a16 = [](const float* q) { return ((uintptr_t)q & 15u) == 0; };
    return c.rbgs_kernel == HNS_RBGS_SPLIT && !(flags & HNS_SOLVE_NEUMANN) && c.topo.num_leaves < (int64_t(1) << 22) &&
           a16(div) && a16(p);
}

// Schedule: iterations 0..K-1 (K even). Check c is evaluated inside iteration
// k_c = (c+1)E - 1 (E even, so k_c is odd) on the iterate that iteration reads; every later
// iteration reads the latest check's slot and returns at once if it passed. Skipping thus
// starts at an even iteration, and the last executed iteration is odd, so with the
// ping-pong order below the result always ends in p.
SolvePlan rbgs_solve_checked(Context& c, const float* div, float* p, int max_iterations, float omega, unsigned flags,
                             double tol, int check_every) {
    SolvePlan plan;
    if (tol <= 0.0) {
        rbgs_solve(c, div, p, max_iterations, omega, flags);
        plan.max_iterations = max_iterations;
        return plan;
    }
    int K = std::max(2, max_iterations + (max_iterations & 1));
    int E = check_every > 0 ? check_every : 10;
    E += E & 1;
    plan.max_iterations = K;
    plan.check_every = E;
    plan.num_checks = K / E;
    plan.tol = tol;
    plan.slots = c.reduce_slots(8 + 2 * std::max(1, plan.num_checks)) + 8;  // first 8 doubles: exact residuals
    HNS_CUDA(cudaMemsetAsync(plan.slots, 0, sizeof(double) * 2 * (size_t)std::max(1, plan.num_checks), c.stream));
    if (use_split32(c, flags, div, p)) {
        split32_solve(c, div, p, K, omega, flags, &plan);
        log_solve(c, plan.slots, plan.num_checks, tol, E, 1, K);
        return plan;
    }
    const size_t n = (size_t)c.num_voxels();
    float* tmp = c.scratch_f32("rbgs_pingpong", n);
    const float* src = (flags & HNS_SOLVE_ZERO_INIT) ? nullptr : p;
    float* buf[2] = {tmp, p};
    const double tol2 = tol * tol;
    for (int it = 0; it < K; ++it) {
        // Latest check completed before iteration `it` (check c runs inside iteration (c+1)E-1).
        const int last_check = it / E - 1;
        const double* chk = last_check >= 0 ? plan.slots + 2 * last_check : nullptr;
        double* out = ((it + 1) % E == 0) ? plan.slots + 2 * ((it + 1) / E - 1) : nullptr;
        float* dst = buf[it & 1];
        launch_rbgs_iteration(c, div, src, dst, omega, flags, chk, tol2, out);
        src = dst;
    }
    log_solve(c, plan.slots, plan.num_checks, tol, E, 1, K);
    return plan;
}

void solve_result(Context& c, const SolvePlan& plan, int* iterations, double* residual) {
    if (plan.num_checks <= 0) {
        *iterations = plan.max_iterations;
        *residual = -1.0;
        return;
    }
    std::vector<double> h(2 * (size_t)plan.num_checks);
    HNS_CUDA(cudaMemcpyAsync(h.data(), plan.slots, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    HNS_CUDA(cudaStreamSynchronize(c.stream));
    const double tol2 = plan.tol * plan.tol;
    for (int q = 0; q < plan.num_checks; ++q) {
        if (h[2 * q] <= tol2 * h[2 * q + 1]) {
            *iterations = (q + 1) * plan.check_every;
            *residual = h[2 * q + 1] > 0 ? std::sqrt(h[2 * q] / h[2 * q + 1]) : 0.0;
            return;
        }
    }
    const int q = plan.num_checks - 1;
    *iterations = plan.max_iterations;
    *residual = h[2 * q + 1] > 0 ? std::sqrt(h[2 * q] / h[2 * q + 1]) : 0.0;
}

namespace {

__global__ void solve_log_kernel(const double* __restrict__ chk, int nchecks, double tol2, int per, int offset,
                                 int cap_iterations, double* __restrict__ log, int cap) {
    int q = nchecks - 1;
    bool hit = false;
    for (int i = 0; i < nchecks; ++i)
        if (chk[2 * i] <= tol2 * chk[2 * i + 1]) {
            q = i;
            hit = true;
            break;
        }
    unsigned long long* count = reinterpret_cast<unsigned long long*>(log + 2 * cap);
    const unsigned long long m = *count;
    double* e = log + 2 * (m % (unsigned long long)cap);
    e[0] = hit ? (double)((q + offset) * per) : (double)cap_iterations;
    e[1] = chk[2 * q + 1] > 0.0 ? sqrt(chk[2 * q] / chk[2 * q + 1]) : 0.0;
    *count = m + 1;
}

}  // namespace

void log_solve(Context& c, const double* checks, int nchecks, double tol, int per, int offset, int cap_iterations) {
    if (nchecks <= 0 || c.d_solve_log.ptr == nullptr) return;
    solve_log_kernel<<<1, 1, 0, c.stream>>>(checks, nchecks, tol * tol, per, offset, cap_iterations,
                                            c.d_solve_log.as<double>(), Context::kSolveLogCap);
    HNS_LAUNCHED();
}

namespace {

double exact_residual(Context& c, const float* div, const float* p, unsigned flags) {
    double* acc = c.reduce_slots(8);
    HNS_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), c.stream));
    launch_residual(c, div, p, acc, flags);
    double h[2];
    HNS_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    HNS_CUDA(cudaStreamSynchronize(c.stream));
    return h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
}

float resolve_omega(const Context& c, float omega) {
    return omega > 0.f ? omega : (float)(2.0f / (1.0f + std::sin(3.14159 * (double)c.dx)));
}

void check_desc(const hns_step_desc* d) {
    if (!d) fail(HNS_ERR_INVALID_ARG, "null step description");
    if (d->max_iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration cap");
    if (d->tolerance < 0.0 || !std::isfinite(d->tolerance)) fail(HNS_ERR_INVALID_ARG, "bad tolerance");
    if (!std::isfinite(d->dt)) fail(HNS_ERR_INVALID_ARG, "bad dt");
}

struct SolveOutcome {
    SolvePlan plan;
    float* div;
    float* p;
    bool refined = false;
    RefinePlan rplan;
};

// Projection of vel (in place): divergence, checked solve from p = 0, gradient subtraction.
SolveOutcome project_in_place(Context& c, float* vel, const hns_step_desc& d) {
    const size_t n = (size_t)c.num_voxels();
    SolveOutcome o;
    o.div = c.scratch_f32("project_div", n);
    o.p = c.scratch_f32("project_p", n);
    if ((d.flags & HNS_SOLVE_NEUMANN) && (d.flags & (HNS_SOLVE_REFINE | HNS_SOLVE_MULTIGRID)))
        fail(HNS_ERR_UNSUPPORTED, "zero-gradient walls are supported by the plain red-black solve only");
    c.phase_begin(HNS_PHASE_DIVERGENCE);
    launch_divergence(c, vel, o.div);
    if (d.flags & HNS_SOLVE_NEUMANN) remove_divergence_mean(c, o.div);  // the singular system's compatibility
    c.phase_end();
    c.phase_begin(HNS_PHASE_SOLVE);
    if (d.flags & HNS_SOLVE_REFINE) {
        if (!(d.tolerance > 0.0)) fail(HNS_ERR_INVALID_ARG, "HNS_SOLVE_REFINE needs a positive tolerance");
        double* p64 = reinterpret_cast<double*>(c.scratch_f32("refine_p", 2 * n));
        o.refined = true;
        o.rplan = refine_solve<float>(c, o.div, p64, d.max_outer > 0 ? d.max_outer : 8,
                                      d.inner_iterations > 0 ? d.inner_iterations : 60, resolve_omega(c, d.omega), d.tolerance,
                                      d.flags);
        c.last_refine = o.rplan;
        c.phase_end();
        c.phase_begin(HNS_PHASE_GRADIENT);
        launch_gradient_f64(c, vel, p64);
        c.phase_end();
        return o;
    }
    o.plan = rbgs_solve_checked(c, o.div, o.p, d.max_iterations, resolve_omega(c, d.omega), d.flags | HNS_SOLVE_ZERO_INIT,
                                d.tolerance, d.check_every);
    c.phase_end();
    c.last_solve = o.plan;
    c.phase_begin(HNS_PHASE_GRADIENT);
    launch_subtract_gradient(c, vel, o.p, vel, nullptr, d.flags);  // pointwise in vel: safe in place
    c.phase_end();
    return o;
}

hns_status finish_info(Context& c, const SolveOutcome& o, const hns_step_desc& d, hns_solve_info* info) {
    if (!info) return HNS_OK;
    if (o.refined) {
        int outer = 0;
        double res = 0.0;
        refine_result(c, o.rplan, &outer, &res);
        info->iterations = outer * o.rplan.inner;
        info->initial_residual = 1.0;
        info->residual = res;
        if (res > d.tolerance)
            return record_error(HNS_ERR_NOT_CONVERGED, "refined solve stopped after " + std::to_string(outer) +
                                                           " outer iterations with residual " + std::to_string(res));
        return HNS_OK;
    }
    int its = 0;
    double chk = 0.0;
    solve_result(c, o.plan, &its, &chk);
    info->iterations = its;
    info->initial_residual = 1.0;
    info->residual = exact_residual(c, o.div, o.p, d.flags);
    if (d.tolerance > 0.0 && info->residual > d.tolerance && chk > d.tolerance)
        return record_error(HNS_ERR_NOT_CONVERGED, "pressure solve stopped at the iteration cap " +
                                                       std::to_string(its) + " with residual " + std::to_string(info->residual));
    return HNS_OK;
}

void set_fields(FieldSet& f, const float* const* in, float* const* out, int base, int count) {
    f.count = count;
    for (int q = 0; q < count; ++q) {
        if (!in[base + q] || !out[base + q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
        if (((uintptr_t)in[base + q] & 3u) != 0 || ((uintptr_t)out[base + q] & 3u) != 0)
            fail(HNS_ERR_INVALID_ARG, "FP32 scalar arrays must be 4-byte aligned");
        f.in[q] = in[base + q];
        f.out[q] = out[base + q];
    }
}

// Advection of velocity and scalars: the first launch carries the velocity and up to
// kMaxAdvectFields scalars; further scalars go in more launches along the same trace.
void advect_chain(Context& c, const float* vel_in, float* vel_out, const float* const* sin, float* const* sout, int ns,
                  float dt) {
    int base = 0;
    c.phase_begin(HNS_PHASE_ADVECT);
    do {
        FieldSet f{};
        set_fields(f, sin, sout, base, std::min(kMaxAdvectFields, ns - base));
        launch_advect_fused(c, vel_in, base == 0 ? vel_out : nullptr, f, dt);
        base += f.count;
    } while (base < ns);
    c.phase_end();
}

}  // namespace

}  // namespace hns

using namespace hns;

extern "C" {

HNS_API hns_status hns_step_plain(hns_ctx* ctx, const float* vel_in, float* vel_out, const float* const* scalars_in,
                                  float* const* scalars_out, int nscalars, const hns_step_desc* desc,
                                  hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        check_desc(desc);
        if (!vel_in || !vel_out) fail(HNS_ERR_INVALID_ARG, "null velocity");
        if (vel_in == vel_out) fail(HNS_ERR_INVALID_ARG, "vel_in and vel_out must differ");
        if (((uintptr_t)vel_in & 3u) != 0 || ((uintptr_t)vel_out & 3u) != 0)
            fail(HNS_ERR_INVALID_ARG, "FP32 velocity arrays must be 4-byte aligned");
        if (nscalars < 0 || (nscalars > 0 && (!scalars_in || !scalars_out))) fail(HNS_ERR_INVALID_ARG, "bad scalar arrays");
        DeviceGuard dg(c->device);
        advect_chain(*c, vel_in, vel_out, scalars_in, scalars_out, nscalars, desc->dt);
        const SolveOutcome o = project_in_place(*c, vel_out, *desc);
        st = finish_info(*c, o, *desc, info);
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_step_plain_host(hns_ctx* ctx, float* vel, float* const* scalars, int nscalars,
                                       const hns_step_desc* desc, hns_solve_info* info) {
    hns_status st = HNS_OK;
    const hns_status g = guarded([&] {
        Context* c = check_ctx(ctx);
        check_desc(desc);
        if (!vel) fail(HNS_ERR_INVALID_ARG, "null velocity");
        if (nscalars < 0 || (nscalars > 0 && !scalars)) fail(HNS_ERR_INVALID_ARG, "bad scalar arrays");
        DeviceGuard dg(c->device);
        const size_t n = (size_t)c->num_voxels();
        float* dv_in = c->scratch_f32("host_vel_in", 3 * n);
        float* dv_out = c->scratch_f32("host_vel_out", 3 * n);
        std::vector<const float*> din((size_t)nscalars);
        std::vector<float*> dout((size_t)nscalars);
        HNS_CUDA(cudaMemcpyAsync(dv_in, vel, 3 * n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        for (int q = 0; q < nscalars; ++q) {
            if (!scalars[q]) fail(HNS_ERR_INVALID_ARG, "null scalar field");
            float* a = c->scratch_f32("host_scalar_in_" + std::to_string(q), n);
            dout[q] = c->scratch_f32("host_scalar_out_" + std::to_string(q), n);
            din[q] = a;
            HNS_CUDA(cudaMemcpyAsync(a, scalars[q], n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        }
        advect_chain(*c, dv_in, dv_out, din.data(), dout.data(), nscalars, desc->dt);
        const SolveOutcome o = project_in_place(*c, dv_out, *desc);
        HNS_CUDA(cudaMemcpyAsync(vel, dv_out, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        for (int q = 0; q < nscalars; ++q)
            HNS_CUDA(cudaMemcpyAsync(scalars[q], dout[q], n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        st = finish_info(*c, o, *desc, info);
    });
    return g != HNS_OK ? g : st;
}

HNS_API hns_status hns_solve_log(hns_ctx* ctx, hns_solve_info* out, int capacity, int* count, int reset) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!count || capacity < 0 || (capacity > 0 && !out)) fail(HNS_ERR_INVALID_ARG, "bad log arguments");
        DeviceGuard dg(c->device);
        const int cap = Context::kSolveLogCap;
        std::vector<double> h(2 * (size_t)cap + 1);
        HNS_CUDA(cudaMemcpyAsync(h.data(), c->d_solve_log.ptr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
        HNS_CUDA(cudaStreamSynchronize(c->stream));
        unsigned long long m = 0;
        std::memcpy(&m, &h[2 * (size_t)cap], sizeof(m));
        *count = (int)std::min<unsigned long long>(m, 0x7fffffffull);
        // The most recent min(m, cap, capacity) entries, oldest first.
        const unsigned long long k = std::min<unsigned long long>({m, (unsigned long long)cap, (unsigned long long)capacity});
        for (unsigned long long q = 0; q < k; ++q) {
            const unsigned long long idx = (m - k + q) % (unsigned long long)cap;
            out[q].iterations = (int)h[2 * idx];
            out[q].residual = h[2 * idx + 1];
            out[q].initial_residual = 1.0;
        }
        if (reset) HNS_CUDA(cudaMemsetAsync(c->d_solve_log.as<double>() + 2 * cap, 0, sizeof(double), c->stream));
    });
}

HNS_API hns_status hns_last_solve(hns_ctx* ctx, hns_solve_info* info) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!info) fail(HNS_ERR_INVALID_ARG, "null info");
        DeviceGuard dg(c->device);
        int its = 0;
        double r = 0.0;
        solve_result(*c, c->last_solve, &its, &r);
        info->iterations = its;
        info->residual = r;
        info->initial_residual = 1.0;
    });
}

}  // extern "C"
