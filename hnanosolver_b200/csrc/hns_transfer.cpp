// Host <-> device copies of field blocks through pinned staging: the transfer boundary of the
// SOP-facing layer (the reference copies each GridIndexedData block with a cudaMemcpyAsync
// from the caller's pageable memory, src/Cuda/HNanoSolver.cu:96-133, 158-221, 471-495).
//
// A copy from or to pageable memory is split into chunks that go through two pinned buffers
// of kChunkBytes. Upload: chunk k is copied from the caller's memory into pinned buffer k % 2
// by several host threads while the DMA of chunk k - 1 runs; download: the DMA of chunk k runs
// while chunk k - 1 is copied out of its pinned buffer. An event per buffer orders its reuse
// after the DMA that read or wrote it. Copies of at most kDirectBytes go directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "hns_internal.cuh"

namespace hns {
namespace {

constexpr size_t kChunkBytes = size_t(64) << 20;
constexpr size_t kDirectBytes = size_t(8) << 20;
constexpr size_t kSliceBytes = size_t(4) << 20;  // smallest share of one host thread

// memcpy split over up to `threads` host threads.
void parallel_copy(void* dst, const void* src, size_t bytes, unsigned threads) {
    const size_t parts = std::max<size_t>(1, std::min<size_t>(threads, bytes / kSliceBytes));
    if (parts == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t per = (bytes + parts - 1) / parts;
    std::vector<std::thread> pool;
    pool.reserve(parts - 1);
    for (size_t q = 1; q < parts; ++q) {
        const size_t off = q * per;
        if (off >= bytes) break;
        pool.emplace_back([=] {
            std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(per, bytes - off));
        });
    }
    std::memcpy(dst, src, std::min(per, bytes));
    for (auto& th : pool) th.join();
}

unsigned copy_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return std::max(1u, std::min(8u, hw));
}

}  // namespace

void Context::ensure_staging() {
    for (int k = 0; k < 2; ++k) {
        if (staging[k] == nullptr) HNS_CUDA(cudaMallocHost(&staging[k], kChunkBytes));
        if (staging_done[k] == nullptr) HNS_CUDA(cudaEventCreateWithFlags(&staging_done[k], cudaEventDisableTiming));
    }
}

void Context::release_staging() {
    for (int k = 0; k < 2; ++k) {
        if (staging_done[k]) (void)cudaEventSynchronize(staging_done[k]);
        if (staging[k]) (void)cudaFreeHost(staging[k]);
        if (staging_done[k]) (void)cudaEventDestroy(staging_done[k]);
        staging[k] = nullptr;
        staging_done[k] = nullptr;
    }
}

void copy_h2d(Context& c, void* dev, const void* host, size_t bytes) {
    if (bytes <= kDirectBytes) {
        HNS_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c.stream));
        HNS_CUDA(cudaStreamSynchronize(c.stream));  // the caller may reuse its buffer on return
        return;
    }
    c.ensure_staging();
    const unsigned threads = copy_threads();
    size_t off = 0;
    for (int k = 0; off < bytes; k ^= 1) {
        const size_t n = std::min(kChunkBytes, bytes - off);
        HNS_CUDA(cudaEventSynchronize(c.staging_done[k]));  // the DMA that last read this buffer is done
        parallel_copy(c.staging[k], static_cast<const char*>(host) + off, n, threads);
        HNS_CUDA(cudaMemcpyAsync(static_cast<char*>(dev) + off, c.staging[k], n, cudaMemcpyHostToDevice, c.stream));
        HNS_CUDA(cudaEventRecord(c.staging_done[k], c.stream));
        off += n;
    }
    HNS_CUDA(cudaStreamSynchronize(c.stream));  // the field is resident when the call returns
}

void copy_d2h(Context& c, void* host, const void* dev, size_t bytes) {
    if (bytes <= kDirectBytes) {
        HNS_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c.stream));
        HNS_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    c.ensure_staging();
    const unsigned threads = copy_threads();
    size_t prev_off = 0, prev_n = 0;
    int prev_k = -1;
    size_t off = 0;
    for (int k = 0; off < bytes || prev_k >= 0; k ^= 1) {
        size_t n = 0;
        if (off < bytes) {
            n = std::min(kChunkBytes, bytes - off);
            HNS_CUDA(cudaEventSynchronize(c.staging_done[k]));
            HNS_CUDA(cudaMemcpyAsync(c.staging[k], static_cast<const char*>(dev) + off, n, cudaMemcpyDeviceToHost, c.stream));
            HNS_CUDA(cudaEventRecord(c.staging_done[k], c.stream));
        }
        if (prev_k >= 0) {  // copy out the previous chunk while this one's DMA runs
            HNS_CUDA(cudaEventSynchronize(c.staging_done[prev_k]));
            parallel_copy(static_cast<char*>(host) + prev_off, c.staging[prev_k], prev_n, threads);
        }
        if (n > 0) {
            prev_k = k, prev_off = off, prev_n = n;
            off += n;
        } else {
            prev_k = -1;
        }
    }
}

}  // namespace hns
