// Inline-PTX helpers for sm_100a: mbarrier-tracked bulk async copies (global -> shared)
// and bounded mbarrier waits. Hand-written from the PTX ISA; no library code.
#pragma once

#include <cstdint>

namespace hns {
namespace ptx {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barrier visible to the async proxy (the bulk-copy engine).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global to
// this CTA's shared memory; completion is counted on `bar` in bytes.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Tiled 4-D tensor load (TMA, no multicast): the box at coordinates (c0, c1, c2, c3), innermost
// first, of the tensor map at `map` (a kernel parameter or global memory) into this CTA's shared
// memory at dst_smem (128-byte aligned); completion is counted on `bar` in bytes. Elements
// outside the tensor arrive as zeros.
__device__ __forceinline__ void tma_load_4d(uint32_t dst_smem, const void* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst_smem),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Asynchronous copy of kBytes (4, 8 or 16; both addresses kBytes-aligned) from global to
// this CTA's shared memory, cached in L1 and L2.
template <int kBytes>
__device__ __forceinline__ void cp_async_ca(void* dst_smem, const void* src_gmem) {
    static_assert(kBytes == 4 || kBytes == 8 || kBytes == 16, "cp.async.ca copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst_smem)), "l"(src_gmem), "n"(kBytes)
                 : "memory");
}

template <int kBytes>
__device__ __forceinline__ void cp_async_ca(uint32_t dst_smem, const void* src_gmem) {
    static_assert(kBytes == 4 || kBytes == 8 || kBytes == 16, "cp.async.ca copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst_smem), "l"(src_gmem), "n"(kBytes) : "memory");
}

// 16-byte asynchronous copy global -> shared cached in L2 only; both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async_cg16(uint32_t dst_smem, const void* src_gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst_smem), "l"(src_gmem) : "memory");
}

// Arrive on `bar` once this thread's earlier cp.async copies have landed. With .noinc the
// arrival counts toward the barrier's expected arrival count (set it at mbarrier.init).
__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy
// (bulk copy) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// try_wait that may suspend the thread for up to `suspend_ns` nanoseconds before returning
// (the hint bounds how long one poll can sleep; the phase completing wakes it earlier).
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t phase, uint32_t suspend_ns) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase), "r"(suspend_ns)
        : "memory");
    return done != 0;
}

// Waits for `phase` of `bar` at most `max_polls` polls (each try_wait itself blocks for a
// hardware-defined interval). Returns false if the wait gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t max_polls) {
    for (uint32_t i = 0; i < max_polls; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// The same with a suspend hint per poll: total wait at most about max_polls * suspend_ns.
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t* bar, uint32_t phase, uint32_t max_polls,
                                                        uint32_t suspend_ns) {
    for (uint32_t i = 0; i < max_polls; ++i)
        if (mbar_try_wait_hint(bar, phase, suspend_ns)) return true;
    return false;
}

// Waits for `phase` of `bar` with try_wait polls (no suspend hint) for at most `max_cycles`
// SM clock cycles. Returns false if the wait gave up.
__device__ __forceinline__ bool mbar_wait_bounded_clock(uint64_t* bar, uint32_t phase, long long max_cycles) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, phase))
        if (clock64() - t0 > max_cycles) return false;
    return true;
}

// The same, but each poll may suspend the thread for up to `suspend_ns` (it resumes as soon as
// the phase completes), so a waiting thread takes no issue slots.
__device__ __forceinline__ bool mbar_wait_bounded_clock_sleep(uint64_t* bar, uint32_t phase, long long max_cycles,
                                                              uint32_t suspend_ns) {
    const long long t0 = clock64();
    while (!mbar_try_wait_hint(bar, phase, suspend_ns))
        if (clock64() - t0 > max_cycles) return false;
    return true;
}

}  // namespace ptx
}  // namespace hns
