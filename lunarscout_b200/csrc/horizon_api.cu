// C-ABI entry points of the horizon march and the slope layout kernels.
#include "internal.cuh"

#include <vector>

namespace ls200 {

// az-major [A, P] -> pixel-major [P, A] through a 32x32 shared tile; with
// `degrees` the value is float32(atanf(s) * float32(180/pi)) and -inf stays
// -inf (contract.py:362-371).
__global__ void __launch_bounds__(256) transpose_kernel(const float *__restrict__ in, int rows,
                                                        int cols, float *__restrict__ out,
                                                        int degrees) {
    __shared__ float tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = in[static_cast<size_t>(r) * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) {
            float v = tile[threadIdx.x][i];
            if (degrees && !isinf(v)) v = __fmul_rn(atanf(v), kSlopeDegrees);
            out[static_cast<size_t>(c) * rows + r] = v;
        }
    }
}

static void launch_transpose(ls200_context *ctx, const float *in, int rows, int cols,
                             float *out, bool degrees) {
    dim3 block(32, 8);
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    transpose_kernel<<<grid, block, 0, ctx->stream>>>(in, rows, cols, out, degrees ? 1 : 0);
    LS_CUDA(cudaGetLastError());
}

void transpose_slopes(ls200_context *ctx, const float *az_major, int azimuth_count,
                      int pixel_count, float *pixel_major, bool degrees) {
    launch_transpose(ctx, az_major, azimuth_count, pixel_count, pixel_major, degrees);
}

void pixel_major_to_az_major(ls200_context *ctx, const float *pixel_major, int azimuth_count,
                             int pixel_count, float *az_major) {
    launch_transpose(ctx, pixel_major, pixel_count, azimuth_count, az_major, false);
}

__global__ void degrees_kernel(const float *__restrict__ in, int64_t n, float *__restrict__ out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const float v = in[i];
        out[i] = isinf(v) && v < 0.0f ? v : __fmul_rn(atanf(v), kSlopeDegrees);
    }
}

// Pixels of a 128x128 pixel-major tile outside the valid (DEM-covered)
// rectangle become -50 degrees, the codec's minimum (file_format.py:93-120).
__global__ void pad_outside_kernel(float *__restrict__ tile, int valid_width, int valid_height,
                                   int azimuth_count) {
    const int pixel = blockIdx.x;
    const int row = pixel / 128, column = pixel % 128;
    if (row < valid_height && column < valid_width) return;
    float *out = tile + static_cast<size_t>(pixel) * azimuth_count;
    for (int a = threadIdx.x; a < azimuth_count; a += blockDim.x) out[a] = -50.0f;
}

void slopes_to_degrees_device(ls200_context *ctx, const float *slopes, int64_t count,
                              float *degrees) {
    const int blocks = static_cast<int>(std::min<int64_t>((count + 255) / 256,
                                                          ctx->props.multiProcessorCount * 16));
    degrees_kernel<<<blocks > 0 ? blocks : 1, 256, 0, ctx->stream>>>(slopes, count, degrees);
    LS_CUDA(cudaGetLastError());
}

// The largest finite s_end (km, field 13) of pass `pass` in host segments
// [A, C, D, 18].
static double host_segment_end_km(const float *segments, int azimuth_count, int center_count,
                                  int dem_count, int pass) {
    double end = 0.0;
    const size_t rays = static_cast<size_t>(azimuth_count) * center_count;
    for (size_t r = 0; r < rays; ++r) {
        const float value = segments[(r * dem_count + pass) * kSegmentFields + 13];
        if (value > end) end = value;  // NaN never compares greater
    }
    return end;
}

static void check_tile(int azimuth_count, int center_count, int dem_count, int tile_width,
                       int tile_height, int subpatch) {
    LS_REQUIRE(azimuth_count > 0 && dem_count > 0, "segment dimensions must be positive");
    LS_REQUIRE(subpatch == 2 || subpatch == 4 || subpatch == 8 || subpatch == 16 ||
                   subpatch == 32 || subpatch == 64 || subpatch == 128,
               "subpatch_size must be a power of two between 2 and 128");
    LS_REQUIRE(tile_width > 0 && tile_height > 0 && tile_width <= 128 && tile_height <= 128,
               "tile dimensions must be between 1 and 128");
    const int count = tile_width / subpatch + 2;
    LS_REQUIRE(center_count == count * count,
               "segment center count does not match tile/subpatch layout");
    LS_REQUIRE(static_cast<int64_t>(tile_width) * tile_height * azimuth_count < (int64_t(1) << 31),
               "tile exceeds the int32 thread index range");
}

void resolve_counters(ls200_context *ctx) {
    if (!ctx->counting) return;
    unsigned long long host[3] = {0, 0, 0};
    LS_CUDA(cudaMemcpyAsync(host, ctx->counters.ptr, sizeof host, cudaMemcpyDeviceToHost,
                            ctx->stream));
    LS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->last_visits = host[0];
    ctx->last_samples = host[1];
    ctx->last_steps = host[2];
}

void reset_counters(ls200_context *ctx) {
    if (ctx->counting)
        LS_CUDA(cudaMemsetAsync(ctx->counters.ptr, 0, 3 * sizeof(unsigned long long),
                                ctx->stream));
}

// All passes on the device; writes pixel-major output into device_out.
static void all_passes_device(ls200_context *ctx, const MarchTile &tile, ls200_dem *const *dems,
                              float *device_out, bool degrees, double *pass_seconds) {
    const int pixel_count = tile.tile_width * tile.tile_height;
    const size_t n = static_cast<size_t>(pixel_count) * tile.azimuth_count;
    ctx->slopes.reserve(n * sizeof(float));
    reset_counters(ctx);
    if (pass_seconds) LS_CUDA(cudaEventRecord(ctx->events[0], ctx->stream));
    for (int pass = 0; pass < tile.dem_count; ++pass) {
        march_pass_device(ctx, tile, dems[0], dems[pass], pass, pass == 0,
                          ctx->slopes.as<float>());
        if (pass_seconds) LS_CUDA(cudaEventRecord(ctx->events[pass + 1], ctx->stream));
    }
    transpose_slopes(ctx, ctx->slopes.as<float>(), tile.azimuth_count, pixel_count, device_out,
                     degrees);
    if (pass_seconds) {
        LS_CUDA(cudaEventSynchronize(ctx->events[tile.dem_count]));
        for (int pass = 0; pass < tile.dem_count; ++pass) {
            float ms = 0.0f;
            LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[pass], ctx->events[pass + 1]));
            pass_seconds[pass] = ms / 1000.0;
        }
    }
    resolve_counters(ctx);
}

}  // namespace ls200

using namespace ls200;

extern "C" {

ls200_status ls200_march_pass(ls200_context *ctx, const float *segments, int azimuth_count,
                              int center_count, int dem_count, const ls200_dem *primary,
                              const ls200_dem *active, int tile_column, int tile_row,
                              int tile_width, int tile_height, int subpatch_size,
                              int pass_index, float observer_elevation_m,
                              const float *slopes_in, float *slopes_out) {
    return guard([&] {
        LS_REQUIRE(ctx && segments && primary && active && slopes_out, "NULL argument");
        check_tile(azimuth_count, center_count, dem_count, tile_width, tile_height,
                   subpatch_size);
        LS_REQUIRE(pass_index >= 0 && pass_index < dem_count,
                   "pass_index is outside the segment DEM axis");
        LS_REQUIRE(active->level_count <= kMaxLevels, "active pyramid is too deep");
        require_march_progress(host_segment_end_km(segments, azimuth_count, center_count,
                                                   dem_count, pass_index),
                               active);
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        const int pixel_count = tile_width * tile_height;
        const size_t n = static_cast<size_t>(pixel_count) * azimuth_count;
        const size_t seg_bytes =
            sizeof(float) * size_t(azimuth_count) * center_count * dem_count * kSegmentFields;
        ctx->segments.reserve(seg_bytes);
        ctx->slopes.reserve(n * sizeof(float));
        ctx->output.reserve(n * sizeof(float));
        LS_CUDA(cudaMemcpyAsync(ctx->segments.ptr, segments, seg_bytes, cudaMemcpyHostToDevice,
                                ctx->stream));
        if (slopes_in) {
            LS_CUDA(cudaMemcpyAsync(ctx->output.ptr, slopes_in, n * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream));
            pixel_major_to_az_major(ctx, ctx->output.as<float>(), azimuth_count, pixel_count,
                                    ctx->slopes.as<float>());
        }
        MarchTile tile{ctx->segments.as<float>(), azimuth_count, center_count, dem_count,
                       tile_column, tile_row, tile_width, tile_height, subpatch_size,
                       observer_elevation_m};
        reset_counters(ctx);
        march_pass_device(ctx, tile, primary, active, pass_index, slopes_in == nullptr,
                          ctx->slopes.as<float>());
        transpose_slopes(ctx, ctx->slopes.as<float>(), azimuth_count, pixel_count,
                         ctx->output.as<float>(), false);
        LS_CUDA(cudaMemcpyAsync(slopes_out, ctx->output.ptr, n * sizeof(float),
                                cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        resolve_counters(ctx);
    });
}

ls200_status ls200_march_all_passes(ls200_context *ctx, const float *segments,
                                    int azimuth_count, int center_count, int dem_count,
                                    ls200_dem *const *dems, int tile_column, int tile_row,
                                    int tile_width, int tile_height, int subpatch_size,
                                    float observer_elevation_m, float *slopes,
                                    double *pass_seconds) {
    return guard([&] {
        LS_REQUIRE(ctx && segments && dems && slopes, "NULL argument");
        check_tile(azimuth_count, center_count, dem_count, tile_width, tile_height,
                   subpatch_size);
        for (int d = 0; d < dem_count; ++d) {
            LS_REQUIRE(dems[d] != nullptr, "NULL DEM");
            require_march_progress(
                host_segment_end_km(segments, azimuth_count, center_count, dem_count, d), dems[d]);
        }
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        const size_t n = static_cast<size_t>(tile_width) * tile_height * azimuth_count;
        const size_t seg_bytes =
            sizeof(float) * size_t(azimuth_count) * center_count * dem_count * kSegmentFields;
        ctx->segments.reserve(seg_bytes);
        ctx->output.reserve(n * sizeof(float));
        LS_CUDA(cudaMemcpyAsync(ctx->segments.ptr, segments, seg_bytes, cudaMemcpyHostToDevice,
                                ctx->stream));
        MarchTile tile{ctx->segments.as<float>(), azimuth_count, center_count, dem_count,
                       tile_column, tile_row, tile_width, tile_height, subpatch_size,
                       observer_elevation_m};
        all_passes_device(ctx, tile, dems, ctx->output.as<float>(), false, pass_seconds);
        LS_CUDA(cudaMemcpyAsync(slopes, ctx->output.ptr, n * sizeof(float),
                                cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_march_all_passes_device(ls200_context *ctx, const float *device_segments,
                                           int azimuth_count, int center_count,
                                           int dem_count, ls200_dem *const *dems,
                                           int tile_column, int tile_row, int tile_width,
                                           int tile_height, int subpatch_size,
                                           float observer_elevation_m, float *device_out,
                                           int degrees, double *pass_seconds) {
    return guard([&] {
        LS_REQUIRE(ctx && device_segments && dems && device_out, "NULL argument");
        check_tile(azimuth_count, center_count, dem_count, tile_width, tile_height,
                   subpatch_size);
        for (int d = 0; d < dem_count; ++d) LS_REQUIRE(dems[d] != nullptr, "NULL DEM");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        MarchTile tile{device_segments, azimuth_count, center_count, dem_count,
                       tile_column, tile_row, tile_width, tile_height, subpatch_size,
                       observer_elevation_m};
        all_passes_device(ctx, tile, dems, device_out, degrees != 0, pass_seconds);
    });
}

ls200_status ls200_horizon_tile(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                                int tile_column, int tile_row, int azimuth_count,
                                double maximum_distance_m, float observer_elevation_m,
                                int subpatch_size, int compress, void *out, int64_t capacity,
                                int64_t *size) {
    return guard([&] {
        LS_REQUIRE(ctx && dems && out && size && dem_count > 0, "NULL argument");
        for (int d = 0; d < dem_count; ++d) LS_REQUIRE(dems[d] != nullptr, "NULL DEM");
        LS_REQUIRE(azimuth_count == 1440 || !compress,
                   "the .cbin tile format holds exactly 1440 azimuths");
        const int tile = 128;
        const int count = tile / subpatch_size + 2;
        check_tile(azimuth_count, count * count, dem_count, tile, tile, subpatch_size);
        const size_t samples = size_t(tile) * tile * azimuth_count;
        const size_t max_payload = size_t(tile) * tile * (2 * 1440 + 2);
        LS_REQUIRE(capacity >= int64_t(compress ? max_payload : samples * sizeof(float)),
                   "output capacity is too small for one tile");
        LS_REQUIRE(tile_column >= 0 && tile_row >= 0, "tile origin must be non-negative");
        const int valid_width = std::min(tile, dems[0]->width - tile_column);
        const int valid_height = std::min(tile, dems[0]->height - tile_row);
        LS_REQUIRE(valid_width > 0 && valid_height > 0, "tile origin lies outside the primary DEM");
        std::unique_lock<std::mutex> hold(ctx->lock);
        activate(ctx);
        const size_t seg_bytes =
            sizeof(float) * size_t(azimuth_count) * count * count * dem_count * kSegmentFields;
        ctx->segments.reserve(seg_bytes);
        ctx->output.reserve(samples * sizeof(float));
        segments_device(ctx, dems, dem_count, tile_column, tile_row, tile, azimuth_count,
                        maximum_distance_m, observer_elevation_m, subpatch_size,
                        ctx->segments.as<float>());
        MarchTile mt{ctx->segments.as<float>(), azimuth_count, count * count, dem_count,
                     tile_column, tile_row, tile, tile, subpatch_size, observer_elevation_m};
        all_passes_device(ctx, mt, dems, ctx->output.as<float>(), true, nullptr);
        if (valid_width < tile || valid_height < tile) {
            pad_outside_kernel<<<tile * tile, 256, 0, ctx->stream>>>(
                ctx->output.as<float>(), valid_width, valid_height, azimuth_count);
            LS_CUDA(cudaGetLastError());
        }
        if (compress) {
            ctx->scratch.reserve(max_payload);
            const int64_t n = cbin_encode(ctx, ctx->output.as<float>(), ctx->scratch.as<uint8_t>());
            LS_CUDA(cudaMemcpyAsync(out, ctx->scratch.ptr, size_t(n), cudaMemcpyDeviceToHost,
                                    ctx->stream));
            *size = n;
        } else {
            LS_CUDA(cudaMemcpyAsync(out, ctx->output.ptr, samples * sizeof(float),
                                    cudaMemcpyDeviceToHost, ctx->stream));
            *size = int64_t(samples * sizeof(float));
        }
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_slopes_to_degrees(ls200_context *ctx, const float *slopes, int64_t count,
                                     float *degrees) {
    return guard([&] {
        LS_REQUIRE(ctx && slopes && degrees, "NULL argument");
        LS_REQUIRE(count >= 0, "count must be non-negative");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        if (count == 0) return;
        ctx->scratch.reserve(2 * sizeof(float) * size_t(count));
        float *d_in = ctx->scratch.as<float>();
        float *d_out = d_in + count;
        LS_CUDA(cudaMemcpyAsync(d_in, slopes, sizeof(float) * count, cudaMemcpyHostToDevice,
                                ctx->stream));
        slopes_to_degrees_device(ctx, d_in, count, d_out);
        LS_CUDA(cudaMemcpyAsync(degrees, d_out, sizeof(float) * count, cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
