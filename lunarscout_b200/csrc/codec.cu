// Horizon tile codec (.cbin) on the device.
//
// Format (src/lunarscout/_numba_horizon/file_format.py:39-73, 135-182): for
// each of the 16384 pixels of a tile, a little-endian u16 block length, then
// the block: the first sample quantised to a big-endian i16, then one delta
// per sample — 7 bits (one byte) when -64 <= d < 63, else 15 bits in two
// bytes with the top bit set.  Samples are degrees clamped to [-50, 50] and
// quantised as round-half-away(float32(value) * float32(32767)/float32(50));
// -inf (pixels outside the DEM) encodes as -50.
//
// Encoding: one thread per pixel writes its block into a fixed 2880-byte
// slot, a single-block scan turns lengths into offsets, and a copy kernel
// packs [length][block] records.  Decoding: the host walks the 16384 length
// prefixes (validating structure) and one thread per pixel expands its block.
#include "internal.cuh"

#include <vector>

namespace ls200 {

constexpr int kCodecPixels = 128 * 128;
constexpr int kCodecSamples = 1440;
constexpr int kMaxBlock = 2 * kCodecSamples;

__device__ __forceinline__ int quantize(float degrees, float short_scale) {
    // max(-50, min(50, v)) in float64 of a float32 is exact, so the clamp
    // can be done in float32; NaN never reaches the encoder.
    float v = degrees < 50.0f ? degrees : 50.0f;
    v = v > -50.0f ? v : -50.0f;
    const double scaled = static_cast<double>(__fmul_rn(v, short_scale));
    const double rounded = scaled >= 0.0 ? floor(scaled + 0.5) : ceil(scaled - 0.5);
    int q = static_cast<int>(rounded);
    return q > 32767 ? 32767 : (q < -32767 ? -32767 : q);
}

__global__ void encode_kernel(const float *__restrict__ degrees, float short_scale,
                              uint8_t *__restrict__ slots, int *__restrict__ lengths) {
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= kCodecPixels) return;
    const float *row = degrees + static_cast<size_t>(pixel) * kCodecSamples;
    uint8_t *out = slots + static_cast<size_t>(pixel) * kMaxBlock;
    int previous = quantize(row[0], short_scale);
    out[0] = static_cast<uint8_t>((previous >> 8) & 0xFF);
    out[1] = static_cast<uint8_t>(previous & 0xFF);
    int n = 2;
    for (int k = 1; k < kCodecSamples; ++k) {
        const int q = quantize(row[k], short_scale);
        int delta = q - previous;
        delta = delta < -16384 ? -16384 : (delta > 16383 ? 16383 : delta);
        previous = ((previous + delta + 32768) & 0xFFFF) - 32768;
        if (delta >= 0 && delta < 63) {
            out[n++] = static_cast<uint8_t>(delta);
        } else if (delta >= -64 && delta < 0) {
            out[n++] = static_cast<uint8_t>(delta & 0x7F);
        } else {
            out[n++] = static_cast<uint8_t>(((delta >> 8) & 0xFF) | 0x80);
            out[n++] = static_cast<uint8_t>(delta & 0xFF);
        }
    }
    lengths[pixel] = n;
}

// Exclusive scan of (2 + length) over the 16384 pixels in one block of 1024
// threads (16 pixels per thread), plus the total.
__global__ void __launch_bounds__(1024) scan_kernel(const int *__restrict__ lengths,
                                                    long long *__restrict__ offsets,
                                                    long long *__restrict__ total) {
    __shared__ long long partial[1024];
    const int t = threadIdx.x;
    long long local[16];
    long long sum = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        local[i] = sum;
        sum += 2 + lengths[t * 16 + i];
    }
    partial[t] = sum;
    __syncthreads();
    for (int stride = 1; stride < 1024; stride <<= 1) {
        const long long add = t >= stride ? partial[t - stride] : 0;
        __syncthreads();
        partial[t] += add;
        __syncthreads();
    }
    const long long before = t == 0 ? 0 : partial[t - 1];
#pragma unroll
    for (int i = 0; i < 16; ++i) offsets[t * 16 + i] = before + local[i];
    if (t == 1023) *total = partial[1023];
}

__global__ void pack_kernel(const uint8_t *__restrict__ slots, const int *__restrict__ lengths,
                            const long long *__restrict__ offsets, uint8_t *__restrict__ payload) {
    // One block per pixel: the record is copied by the block's threads.
    const int pixel = blockIdx.x;
    const int n = lengths[pixel];
    uint8_t *dst = payload + offsets[pixel];
    if (threadIdx.x == 0) {
        dst[0] = static_cast<uint8_t>(n & 0xFF);
        dst[1] = static_cast<uint8_t>((n >> 8) & 0xFF);
    }
    const uint8_t *src = slots + static_cast<size_t>(pixel) * kMaxBlock;
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[2 + i] = src[i];
}

__global__ void decode_kernel(const uint8_t *__restrict__ payload,
                              const long long *__restrict__ block_start,
                              const int *__restrict__ lengths, float elevation_scale,
                              float *__restrict__ degrees, int *__restrict__ error) {
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= kCodecPixels) return;
    const uint8_t *p = payload + block_start[pixel];
    const int n = lengths[pixel];
    float *row = degrees + static_cast<size_t>(pixel) * kCodecSamples;
    int accumulator = (static_cast<int>(p[0]) << 8) | p[1];
    if (accumulator >= 32768) accumulator -= 65536;
    row[0] = __fmul_rn(static_cast<float>(accumulator), elevation_scale);
    int offset = 2, k = 1;
    while (offset < n && k < kCodecSamples) {
        const int first = p[offset++];
        int delta;
        if (first & 0x80) {
            if (offset >= n) break;
            const int high = ((first << 1) & 0x80) | (first & 0x7F);
            delta = (high << 8) | p[offset++];
            if (delta >= 32768) delta -= 65536;
        } else {
            delta = first & 0x7F;
            if (delta & 0x40) delta -= 0x80;
        }
        accumulator = ((accumulator + delta + 32768) & 0xFFFF) - 32768;
        row[k++] = __fmul_rn(static_cast<float>(accumulator), elevation_scale);
    }
    if (k != kCodecSamples || offset != n) atomicExch(error, pixel + 1);
}

static float short_scale() { return 32767.0f / 50.0f; }
static float elevation_scale() { return 50.0f / 32767.0f; }

struct CodecBuffers {
    DeviceBuffer slots, lengths, offsets, total, payload, degrees, error;
};

static CodecBuffers &codec_buffers(ls200_context *ctx) {
    if (!ctx->codec) ctx->codec = new CodecBuffers();
    return *ctx->codec;
}

void release_codec(ls200_context *ctx) {
    delete ctx->codec;
    ctx->codec = nullptr;
}

// Encode device degrees [16384, 1440] into device `payload` (capacity at
// least 16384 * 2882); returns the payload size (synchronises).
int64_t cbin_encode(ls200_context *ctx, const float *degrees, uint8_t *payload) {
    CodecBuffers &b = codec_buffers(ctx);
    b.slots.reserve(size_t(kCodecPixels) * kMaxBlock);
    b.lengths.reserve(sizeof(int) * kCodecPixels);
    b.offsets.reserve(sizeof(long long) * kCodecPixels);
    b.total.reserve(sizeof(long long));
    encode_kernel<<<kCodecPixels / 128, 128, 0, ctx->stream>>>(degrees, short_scale(),
                                                               b.slots.as<uint8_t>(),
                                                               b.lengths.as<int>());
    LS_CUDA(cudaGetLastError());
    scan_kernel<<<1, 1024, 0, ctx->stream>>>(b.lengths.as<int>(), b.offsets.as<long long>(),
                                             b.total.as<long long>());
    LS_CUDA(cudaGetLastError());
    pack_kernel<<<kCodecPixels, 128, 0, ctx->stream>>>(b.slots.as<uint8_t>(), b.lengths.as<int>(),
                                                       b.offsets.as<long long>(), payload);
    LS_CUDA(cudaGetLastError());
    long long total = 0;
    LS_CUDA(cudaMemcpyAsync(&total, b.total.ptr, sizeof total, cudaMemcpyDeviceToHost,
                            ctx->stream));
    LS_CUDA(cudaStreamSynchronize(ctx->stream));
    return total;
}

}  // namespace ls200

using namespace ls200;

extern "C" {

ls200_status ls200_cbin_encode_device(ls200_context *ctx, const float *device_degrees,
                                      uint8_t *device_payload, int64_t *size) {
    return guard([&] {
        LS_REQUIRE(ctx && device_degrees && device_payload && size, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        *size = cbin_encode(ctx, device_degrees, device_payload);
    });
}

ls200_status ls200_cbin_encode(ls200_context *ctx, const float *degrees, uint8_t *payload,
                               int64_t capacity, int64_t *size) {
    return guard([&] {
        LS_REQUIRE(ctx && degrees && payload && size, "NULL argument");
        LS_REQUIRE(capacity >= int64_t(kCodecPixels) * (kMaxBlock + 2),
                   "payload capacity must be at least 16384 * 2882 bytes");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        CodecBuffers &b = codec_buffers(ctx);
        const size_t n = sizeof(float) * size_t(kCodecPixels) * kCodecSamples;
        b.degrees.reserve(n);
        b.payload.reserve(size_t(kCodecPixels) * (kMaxBlock + 2));
        LS_CUDA(cudaMemcpyAsync(b.degrees.ptr, degrees, n, cudaMemcpyHostToDevice, ctx->stream));
        const int64_t total = cbin_encode(ctx, b.degrees.as<float>(), b.payload.as<uint8_t>());
        LS_CUDA(cudaMemcpyAsync(payload, b.payload.ptr, size_t(total), cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        *size = total;
    });
}

ls200_status ls200_cbin_decode(ls200_context *ctx, const uint8_t *payload, int64_t size,
                               float *degrees) {
    return guard([&] {
        LS_REQUIRE(ctx && payload && degrees && size >= 0, "invalid arguments");
        // Structure (file_format.py:135-182): 16384 records, each a u16 LE
        // length in [2, 2880] followed by that many bytes, and no trailing
        // bytes.
        std::vector<long long> starts(kCodecPixels);
        std::vector<int> lengths(kCodecPixels);
        long long offset = 0;
        for (int p = 0; p < kCodecPixels; ++p) {
            LS_REQUIRE(offset + 2 <= size, "compressed horizon ended while reading a block length");
            const int length = payload[offset] | (payload[offset + 1] << 8);
            offset += 2;
            LS_REQUIRE(length >= 2 && length <= kMaxBlock, "compressed horizon block length is invalid");
            LS_REQUIRE(offset + length <= size, "compressed horizon ended inside a block");
            starts[p] = offset;
            lengths[p] = length;
            offset += length;
        }
        LS_REQUIRE(offset == size, "compressed horizon contains trailing bytes");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        CodecBuffers &b = codec_buffers(ctx);
        const size_t n = sizeof(float) * size_t(kCodecPixels) * kCodecSamples;
        b.payload.reserve(size_t(size) > 0 ? size_t(size) : 1);
        b.offsets.reserve(sizeof(long long) * kCodecPixels);
        b.lengths.reserve(sizeof(int) * kCodecPixels);
        b.degrees.reserve(n);
        b.error.reserve(sizeof(int));
        LS_CUDA(cudaMemcpyAsync(b.payload.ptr, payload, size_t(size), cudaMemcpyHostToDevice,
                                ctx->stream));
        LS_CUDA(cudaMemcpyAsync(b.offsets.ptr, starts.data(), sizeof(long long) * kCodecPixels,
                                cudaMemcpyHostToDevice, ctx->stream));
        LS_CUDA(cudaMemcpyAsync(b.lengths.ptr, lengths.data(), sizeof(int) * kCodecPixels,
                                cudaMemcpyHostToDevice, ctx->stream));
        LS_CUDA(cudaMemsetAsync(b.error.ptr, 0, sizeof(int), ctx->stream));
        decode_kernel<<<kCodecPixels / 128, 128, 0, ctx->stream>>>(
            b.payload.as<uint8_t>(), b.offsets.as<long long>(), b.lengths.as<int>(),
            elevation_scale(), b.degrees.as<float>(), b.error.as<int>());
        LS_CUDA(cudaGetLastError());
        int error = 0;
        LS_CUDA(cudaMemcpyAsync(&error, b.error.ptr, sizeof error, cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaMemcpyAsync(degrees, b.degrees.ptr, n, cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        LS_REQUIRE(error == 0, "compressed horizon block did not decode to 1440 samples");
    });
}

}  // extern "C"
