// qm_transfer.cpp -- whole-state copies between a caller's host buffer and the device.
//
// The drop-in port receives the amplitudes as the caller's own array: for the .NET shim a
// pinned managed Complex[] (pinned against the garbage collector, not page-locked), for Python
// a numpy array.  cudaMemcpy from such pageable memory goes through the driver's own small
// bounce buffers: on the B200 host a 16 GiB state moves at about 6 GiB/s each way, a quarter
// of a page-locked buffer's rate.  Here a large pageable copy moves through two 64 MiB
// page-locked bounce buffers of the context instead: host threads fill (or drain) one while
// the copy engine moves the other.  Page-locked buffers (cudaHostAlloc, cudaHostRegister,
// qm_host_alloc) and small copies go straight to the copy engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "qm_internal.h"

namespace {

constexpr size_t kBounceBytes = size_t(64) << 20;
constexpr size_t kStagedMin = size_t(16) << 20;  // smaller copies go straight to the copy engine

bool page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

// memcpy split over a few host threads (one thread does not saturate host memory bandwidth)
void parallel_copy(void* dst, const void* src, size_t n) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t workers = std::min<size_t>({8, std::max<size_t>(1, hw / 2), std::max<size_t>(1, n >> 22)});
    if (workers <= 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t slice = ((n + workers - 1) / workers + 63) & ~size_t(63);
    std::vector<std::thread> pool;
    for (size_t w = 1; w < workers; ++w) {
        const size_t b = w * slice;
        if (b >= n) break;
        pool.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + b, static_cast<const char*>(src) + b, std::min(slice, n - b)); });
    }
    std::memcpy(dst, src, std::min(slice, n));
    for (auto& t : pool) t.join();
}

cudaError_t ensure_bounce(qm_context* ctx) {
    for (int i = 0; i < 2; ++i) {
        if (!ctx->bounce[i]) {
            cudaError_t e = cudaHostAlloc(&ctx->bounce[i], kBounceBytes, cudaHostAllocDefault);
            if (e != cudaSuccess) return e;
        }
        if (!ctx->bounce_done[i]) {
            cudaError_t e = cudaEventCreateWithFlags(&ctx->bounce_done[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t host_to_device(qm_context* ctx, void* dev, const void* host, size_t bytes) {
    if (bytes < kStagedMin || page_locked(host))
        return cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaError_t e = ensure_bounce(ctx);
    if (e != cudaSuccess) return e;
    for (size_t off = 0, i = 0; off < bytes; off += kBounceBytes, ++i) {
        const int b = (int)(i & 1);
        const size_t n = std::min(kBounceBytes, bytes - off);
        if ((e = cudaEventSynchronize(ctx->bounce_done[b])) != cudaSuccess) return e;  // its last copy is done
        parallel_copy(ctx->bounce[b], static_cast<const char*>(host) + off, n);
        if ((e = cudaMemcpyAsync(static_cast<char*>(dev) + off, ctx->bounce[b], n, cudaMemcpyHostToDevice,
                                 ctx->stream)) != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ctx->bounce_done[b], ctx->stream)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t device_to_host(qm_context* ctx, void* host, const void* dev, size_t bytes) {
    cudaError_t e;
    if (bytes < kStagedMin || page_locked(host)) {
        e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        return e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
    }
    if ((e = ensure_bounce(ctx)) != cudaSuccess) return e;
    const size_t chunks = (bytes + kBounceBytes - 1) / kBounceBytes;
    auto issue = [&](size_t i) -> cudaError_t {
        const int b = (int)(i & 1);
        const size_t off = i * kBounceBytes, n = std::min(kBounceBytes, bytes - off);
        cudaError_t r = cudaMemcpyAsync(ctx->bounce[b], static_cast<const char*>(dev) + off, n, cudaMemcpyDeviceToHost,
                                        ctx->stream);
        return r == cudaSuccess ? cudaEventRecord(ctx->bounce_done[b], ctx->stream) : r;
    };
    for (size_t i = 0; i < std::min<size_t>(2, chunks); ++i)
        if ((e = issue(i)) != cudaSuccess) return e;
    for (size_t i = 0; i < chunks; ++i) {
        const int b = (int)(i & 1);
        const size_t off = i * kBounceBytes, n = std::min(kBounceBytes, bytes - off);
        if ((e = cudaEventSynchronize(ctx->bounce_done[b])) != cudaSuccess) return e;
        parallel_copy(static_cast<char*>(host) + off, ctx->bounce[b], n);
        if (i + 2 < chunks && (e = issue(i + 2)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void release_bounce(qm_context* ctx) {
    for (int i = 0; i < 2; ++i) {
        if (ctx->bounce[i]) cudaFreeHost(ctx->bounce[i]);
        if (ctx->bounce_done[i]) cudaEventDestroy(ctx->bounce_done[i]);
        ctx->bounce[i] = nullptr;
        ctx->bounce_done[i] = nullptr;
    }
}
