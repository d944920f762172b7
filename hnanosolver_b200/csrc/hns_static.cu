// hns_project_static: the projection of hns_project (divergence, zero-initialised red-black
// solve, gradient subtraction; src/Cuda/PressureProjection.cu:9-78) with its solver scratch in
// one fixed device array compiled into this file instead of context-owned allocations. The
// call allocates nothing: no cudaMalloc, no cudaFree, no allocating library routine.
//
// The array lives in this translation unit only, so under CUDA's lazy module loading it
// occupies device memory only in processes that call hns_project_static.
#include <cstdint>
#include <mutex>

#include "hns_internal.cuh"

namespace hns {
namespace {

// At most 2^20 active voxels (2048 leaves); three FP32 arrays of that size: 12 MiB.
constexpr size_t kStaticMaxVoxels = size_t(1) << 20;
constexpr int kStaticMaxDevices = 64;

// [0, M): divergence; [M, 2M): pressure; [2M, 3M): red-black ping-pong buffer (M = kStaticMaxVoxels).
static __device__ __align__(256) float g_static_scratch[3 * kStaticMaxVoxels];

std::mutex g_static_mu;
float* g_static_ptr[kStaticMaxDevices] = {};

// Address of g_static_scratch on `device`, with that device current (the caller holds a
// DeviceGuard for it). The first lookup also loads this file's module. Outside stream capture
// the address is looked up again on every call (cheap), so a primary context that was reset and
// re-created in between gets the array's new address; while the stream is being captured the
// address cached by an earlier call is used, so that the first call must come before capture.
float* static_scratch(int device, cudaStream_t stream) {
    if (device < 0 || device >= kStaticMaxDevices)
        fail(HNS_ERR_UNSUPPORTED, "hns_project_static supports device ordinals below " + std::to_string(kStaticMaxDevices));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    HNS_CUDA(cudaStreamIsCapturing(stream, &cap));
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (cap == cudaStreamCaptureStatusNone || !g_static_ptr[device]) {
        float* ptr = nullptr;
        HNS_CUDA(cudaGetSymbolAddress((void**)&ptr, g_static_scratch));
        g_static_ptr[device] = ptr;
    }
    return g_static_ptr[device];
}

}  // namespace
}  // namespace hns

using namespace hns;

extern "C" {

HNS_API hns_status hns_project_static(hns_ctx* ctx, float* vel, int iterations, float omega, unsigned flags,
                                      hns_solve_info* info) {
    return guarded([&] {
        Context* c = check_ctx(ctx);
        if (!vel) fail(HNS_ERR_INVALID_ARG, "null velocity");
        if (((uintptr_t)vel & 3u) != 0) fail(HNS_ERR_INVALID_ARG, "velocity must be 4-byte aligned");
        if (iterations < 0) fail(HNS_ERR_INVALID_ARG, "negative iteration count");
        if (flags & HNS_SOLVE_NEUMANN)
            fail(HNS_ERR_UNSUPPORTED, "hns_project_static takes the reference's walls only (its component sums would allocate)");
        const size_t n = (size_t)c->num_voxels();
        if (n > kStaticMaxVoxels)
            fail(HNS_ERR_UNSUPPORTED, "hns_project_static: the grid has " + std::to_string(n) +
                                          " active voxels, above the fixed scratch's maximum of " +
                                          std::to_string(kStaticMaxVoxels) + " (2048 leaves); use hns_project");
        DeviceGuard g(c->device);
        float* base = static_scratch(c->device, c->stream);
        float* div = base;
        float* p = base + kStaticMaxVoxels;
        float* tmp = base + 2 * kStaticMaxVoxels;
        if (!(omega > 0.f)) omega = (float)(2.0f / (1.0f + std::sin(3.14159 * (double)c->dx)));
        launch_divergence(*c, vel, div);
        // The pressure starts at zero: the initial residual reads it, a zero-iteration solve
        // returns it, and an earlier call's pressure must not leak into this one.
        HNS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(float), c->stream));
        double* acc = nullptr;
        if (info) {
            acc = c->reduce_slots(4);  // allocated when the context was created
            HNS_CUDA(cudaMemsetAsync(acc, 0, 4 * sizeof(double), c->stream));
            launch_residual(*c, div, p, acc, flags);
        }
        // Zero-initialised ping-pong: the first iteration reads p = 0 implicitly and the last
        // one writes into p.
        const float* src = nullptr;
        for (int it = 0; it < iterations; ++it) {
            float* dst = ((iterations - it) & 1) ? p : tmp;
            launch_rbgs_iteration(*c, div, src, dst, omega, flags);
            src = dst;
        }
        if (info) launch_residual(*c, div, p, acc + 2, flags);
        launch_subtract_gradient(*c, vel, p, vel);
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
