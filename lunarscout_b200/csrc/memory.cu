// Pinned host buffers, device-allocation accounting and the FP32-issue
// reference probe of the ls200 C ABI.
#include <unordered_map>

#include "internal.cuh"

namespace ls200 {

namespace {
constexpr int kTrackedDevices = 64;
std::mutex g_memory_lock;
std::unordered_map<void *, std::pair<int, size_t>> g_allocations;
int64_t g_in_use[kTrackedDevices] = {};
int64_t g_peak[kTrackedDevices] = {};
}  // namespace

cudaError_t tracked_malloc_bytes(void **ptr, size_t bytes) {
    const cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) return e;
    int device = 0;
    cudaGetDevice(&device);
    if (device < 0 || device >= kTrackedDevices) device = 0;
    std::lock_guard<std::mutex> hold(g_memory_lock);
    g_allocations[*ptr] = {device, bytes};
    g_in_use[device] += static_cast<int64_t>(bytes);
    if (g_in_use[device] > g_peak[device]) g_peak[device] = g_in_use[device];
    return e;
}

cudaError_t tracked_free(void *ptr) {
    if (!ptr) return cudaSuccess;
    {
        std::lock_guard<std::mutex> hold(g_memory_lock);
        const auto found = g_allocations.find(ptr);
        if (found != g_allocations.end()) {
            g_in_use[found->second.first] -= static_cast<int64_t>(found->second.second);
            g_allocations.erase(found);
        }
    }
    return cudaFree(ptr);
}

// 8 independent FMA chains per thread: the issue-rate ceiling of the FP32
// pipe, used as the measured denominator of the march roofline (the driver's
// peak table has HBM and tensor figures but no FP32 one).
__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int iterations, float seed) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = __fmaf_rn(a0, m, c); a1 = __fmaf_rn(a1, m, c);
            a2 = __fmaf_rn(a2, m, c); a3 = __fmaf_rn(a3, m, c);
            a4 = __fmaf_rn(a4, m, c); a5 = __fmaf_rn(a5, m, c);
            a6 = __fmaf_rn(a6, m, c); a7 = __fmaf_rn(a7, m, c);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678f) out[0] = r;  // keeps the chains live
}

}  // namespace ls200

using namespace ls200;

extern "C" {

ls200_status ls200_host_alloc(int64_t bytes, void **out) {
    return guard([&] {
        LS_REQUIRE(out != nullptr && bytes >= 0, "invalid allocation request");
        *out = nullptr;
        if (bytes == 0) return;
        LS_CUDA(cudaHostAlloc(out, static_cast<size_t>(bytes), cudaHostAllocPortable));
    });
}

ls200_status ls200_host_free(void *ptr) {
    return guard([&] {
        if (ptr) LS_CUDA(cudaFreeHost(ptr));
    });
}

ls200_status ls200_memory_stats(int device, int64_t *in_use, int64_t *peak, int reset_peak) {
    return guard([&] {
        LS_REQUIRE(device >= 0 && device < kTrackedDevices, "device index out of range");
        std::lock_guard<std::mutex> hold(g_memory_lock);
        if (in_use) *in_use = g_in_use[device];
        if (peak) *peak = g_peak[device];
        if (reset_peak) g_peak[device] = g_in_use[device];
    });
}

ls200_status ls200_fp32_probe(ls200_context *ctx, int iterations, double *tflops) {
    return guard([&] {
        LS_REQUIRE(ctx && tflops && iterations > 0, "invalid probe request");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        ctx->scratch.reserve(sizeof(float));
        const int blocks = ctx->props.multiProcessorCount * 8;
        fma_probe_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->scratch.as<float>(), 8, 1.0f);
        LS_CUDA(cudaGetLastError());
        LS_CUDA(cudaEventRecord(ctx->events[0], ctx->stream));
        fma_probe_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->scratch.as<float>(), iterations,
                                                          1.0f);
        LS_CUDA(cudaGetLastError());
        LS_CUDA(cudaEventRecord(ctx->events[1], ctx->stream));
        LS_CUDA(cudaEventSynchronize(ctx->events[1]));
        float ms = 0.f;
        LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
        const double flops = 2.0 * 8 * 16 * double(iterations) * blocks * 256;
        *tflops = flops / (ms * 1e-3) / 1e12;
    });
}

}  // extern "C"
