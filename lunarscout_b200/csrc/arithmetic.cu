// Exhaustive check of the march's correctly rounded reciprocal
// (reciprocal_pair in march_core.cuh: hardware approximation plus one
// Newton-Raphson step) against the IEEE sequence __frcp_rn, bit for bit, on
// every 32-bit pattern with |x| >= 2^-64 (the march uses it for |x| > 1e-8).
// The march's bit parity with the reference rests on it; a GPU test and the
// smoke check run it on the device the march runs on.
#include "march_core.cuh"

namespace ls200 {

// Grid-stride over the patterns 2^-64 <= |x| (infinities and NaN included),
// each through both lanes with both signs: (x, -x).
__global__ void arithmetic_check_kernel(unsigned long long *counts) {
    constexpr unsigned kFirst = (127u - 64u) << 23;  // 2^-64
    constexpr unsigned long long kCount = 0x80000000ull - kFirst;
    unsigned long long mismatches = 0;
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x +
                                threadIdx.x;
         i < kCount; i += stride) {
        const float x = __uint_as_float(kFirst + static_cast<unsigned>(i));
        const float2 paired = reciprocal_pair(pair(x, -x));
        mismatches += __float_as_uint(paired.x) != __float_as_uint(__frcp_rn(x));
        mismatches += __float_as_uint(paired.y) != __float_as_uint(__frcp_rn(-x));
    }
    if (mismatches) atomicAdd(counts, mismatches);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(counts + 1, 2 * kCount);
}

}  // namespace ls200

using namespace ls200;

extern "C" ls200_status ls200_check_arithmetic(ls200_context *ctx, int64_t *mismatches,
                                               int64_t *checked) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context must not be NULL");
        activate(ctx);
        std::lock_guard<std::mutex> hold(ctx->lock);
        DeviceBuffer counts;
        counts.reserve(2 * sizeof(unsigned long long));
        LS_CUDA(cudaMemsetAsync(counts.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
        arithmetic_check_kernel<<<static_cast<unsigned>(ctx->props.multiProcessorCount) * 16, 256,
                                  0, ctx->stream>>>(counts.as<unsigned long long>());
        LS_CUDA(cudaGetLastError());
        unsigned long long host[2] = {0, 0};
        LS_CUDA(cudaMemcpyAsync(host, counts.ptr, sizeof host, cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (mismatches) *mismatches = static_cast<int64_t>(host[0]);
        if (checked) *checked = static_cast<int64_t>(host[1]);
    });
}
