// Context lifecycle, error plumbing and device-resident DEMs of the ls200 C ABI.
#include "internal.cuh"

#include <cmath>
#include <vector>

namespace ls200 {

static thread_local std::string g_last_error;

void set_last_error(const std::string &message) { g_last_error = message; }

void activate(ls200_context *ctx) { LS_CUDA(cudaSetDevice(ctx->device)); }

int pyramid_layout(int width, int height, PyramidLevel *levels, int capacity,
                   int64_t *mip_count) {
    // Factor-four levels down to 1x1 (pyramid.py:19-31): level 0 has offset 0,
    // mip levels are packed back to back.
    int count = 0;
    int64_t offset = 0;
    int w = width, h = height;
    for (;;) {
        if (levels && count < capacity) {
            levels[count].offset = count == 0 ? 0 : static_cast<int>(offset);
            levels[count].width = w;
            levels[count].height = h;
        }
        if (count > 0) offset += static_cast<int64_t>(w) * h;
        ++count;
        if (w == 1 && h == 1) break;
        w = (w + 3) / 4;
        h = (h + 3) / 4;
    }
    if (mip_count) *mip_count = offset;
    return count;
}

double dem_resolution_m(const ls200_dem *dem) {
    const float *m = dem->map_parameters;
    return 0.5 * (std::hypot(double(m[6]), double(m[9])) + std::hypot(double(m[7]), double(m[10])));
}

void require_march_progress(double s_end_km, const ls200_dem *active) {
    if (!(s_end_km > 0.0)) return;  // no segment reaches past its start
    LS_REQUIRE(s_end_km < 2048.0,
               "rays longer than 2048 km cannot be marched in FP32 (the position would stop "
               "moving)");
    int exponent = 0;
    std::frexp(s_end_km, &exponent);  // s_end_km = f * 2^exponent, f in [0.5, 1)
    const double ulp_km = std::ldexp(1.0, exponent - 24);
    const double resolution = dem_resolution_m(active);
    LS_REQUIRE(std::isfinite(resolution) && resolution * 0.5e-3 > 2.0 * ulp_km,
               "the DEM's pixel size is too small for rays of this length (the FP32 position "
               "would stop moving)");
}

}  // namespace ls200

using namespace ls200;

extern "C" {

const char *ls200_last_error(void) { return g_last_error.c_str(); }

int ls200_abi_version(void) { return 1; }

ls200_status ls200_context_create(int device_id, ls200_context **out) {
    return guard([&] {
        LS_REQUIRE(out != nullptr, "out must not be NULL");
        *out = nullptr;
        int count = 0;
        cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0) {
            cudaGetLastError();
            throw Error(LS200_ERR_UNAVAILABLE,
                        std::string("no CUDA device is visible: ") + cudaGetErrorString(e));
        }
        if (device_id < 0 || device_id >= count)
            throw Error(LS200_ERR_UNAVAILABLE, "cannot select CUDA device " +
                                                   std::to_string(device_id));
        auto ctx = new ls200_context();
        ctx->device = device_id;
        try {
            LS_CUDA(cudaSetDevice(device_id));
            LS_CUDA(cudaGetDeviceProperties(&ctx->props, device_id));
            if (ctx->props.major != 10)
                throw Error(LS200_ERR_UNAVAILABLE,
                            std::string("device ") + ctx->props.name +
                                " is not an sm_100 (Blackwell datacenter) GPU; this "
                                "library is built for sm_100a only");
            LS_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
            ctx->stream = ctx->own_stream;
            for (auto &event : ctx->events) LS_CUDA(cudaEventCreate(&event));
            ctx->counters.reserve(3 * sizeof(unsigned long long));
        } catch (...) {
            for (auto &event : ctx->events)
                if (event) cudaEventDestroy(event);
            if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
            delete ctx;
            throw;
        }
        *out = ctx;
    });
}

ls200_status ls200_context_destroy(ls200_context *ctx) {
    return guard([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        // DEMs still alive belong to this context: release them with it.
        for (ls200_dem *dem : ctx->dems) {
            if (dem->level0) tracked_free(dem->level0);
            if (dem->cells) tracked_free(dem->cells);
            if (dem->bounds) tracked_free(dem->bounds);
            delete dem;
        }
        ctx->dems.clear();
        release_lighting_state(ctx);
        release_codec(ctx);
        release_adjoint_state(ctx);
        for (auto &event : ctx->events)
            if (event) cudaEventDestroy(event);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        delete ctx;
    });
}

ls200_status ls200_device_info(ls200_context *ctx, char *name, int name_capacity, int *major,
                               int *minor, int *sm_count) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        if (name && name_capacity > 0) {
            std::strncpy(name, ctx->props.name, name_capacity - 1);
            name[name_capacity - 1] = '\0';
        }
        if (major) *major = ctx->props.major;
        if (minor) *minor = ctx->props.minor;
        if (sm_count) *sm_count = ctx->props.multiProcessorCount;
    });
}

ls200_status ls200_set_stream(ls200_context *ctx, void *stream) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        std::lock_guard<std::mutex> hold(ctx->lock);
        ctx->stream = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
    });
}

ls200_status ls200_reset_stream(ls200_context *ctx) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        std::lock_guard<std::mutex> hold(ctx->lock);
        ctx->stream = ctx->own_stream;
    });
}

ls200_status ls200_synchronize(ls200_context *ctx) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        activate(ctx);
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_pyramid_layout(int width, int height, int32_t *levels, int capacity,
                                  int *level_count, int64_t *mip_count) {
    return guard([&] {
        LS_REQUIRE(width > 0 && height > 0, "DEM dimensions must be positive");
        PyramidLevel table[kMaxLevels];
        int64_t mips = 0;
        int count = pyramid_layout(width, height, table, kMaxLevels, &mips);
        LS_REQUIRE(count <= kMaxLevels, "DEM is too large for the pyramid table");
        if (levels) {
            for (int l = 0; l < count && l < capacity; ++l) {
                levels[4 * l + 0] = l;
                levels[4 * l + 1] = table[l].offset;
                levels[4 * l + 2] = table[l].width;
                levels[4 * l + 3] = table[l].height;
            }
        }
        if (level_count) *level_count = count;
        if (mip_count) *mip_count = mips;
    });
}

ls200_status ls200_dem_create(ls200_context *ctx, const float *level0, int width, int height,
                              const float *mips, const double *geo_transform,
                              const double *projection, const float *map_parameters,
                              ls200_dem **out) {
    return guard([&] {
        LS_REQUIRE(ctx && level0 && geo_transform && projection && map_parameters && out,
                   "NULL argument");
        LS_REQUIRE(width > 0 && height > 0, "DEM dimensions must be positive");
        LS_REQUIRE(static_cast<int64_t>(width) * height < (int64_t(1) << 31),
                   "DEM exceeds the int32 index range");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        auto dem = new ls200_dem();
        try {
            dem->ctx = ctx;
            dem->width = width;
            dem->height = height;
            dem->level_count =
                pyramid_layout(width, height, dem->levels, kMaxLevels, &dem->mip_count);
            LS_REQUIRE(dem->level_count <= kMaxLevels, "DEM is too large");
            std::memcpy(dem->geo_transform, geo_transform, sizeof dem->geo_transform);
            std::memcpy(dem->projection, projection, sizeof dem->projection);
            std::memcpy(dem->map_parameters, map_parameters, sizeof dem->map_parameters);
            const size_t cells0 = size_t(width) * height;
            LS_REQUIRE(cells0 + size_t(dem->mip_count) < (size_t(1) << 31),
                       "DEM pyramid exceeds the int32 cell index range");
            LS_CUDA(tracked_malloc(&dem->level0, sizeof(float) * cells0));
            // One allocation: sanitized level 0 followed by the packed mips.
            LS_CUDA(tracked_malloc(&dem->cells, sizeof(float) * (cells0 + size_t(dem->mip_count))));
            LS_CUDA(tracked_malloc(&dem->bounds, sizeof(float) * (cells0 + size_t(dem->mip_count))));
            dem->mips = dem->cells + cells0;
            LS_CUDA(cudaMemcpyAsync(dem->level0, level0, sizeof(float) * cells0,
                                    cudaMemcpyHostToDevice, ctx->stream));
            if (mips) {
                LS_CUDA(cudaMemcpyAsync(dem->mips, mips, sizeof(float) * dem->mip_count,
                                        cudaMemcpyHostToDevice, ctx->stream));
            } else {
                build_pyramid_device(ctx, dem);
            }
            sanitize_level0(ctx, dem);
            build_cell_bounds(ctx, dem);
            LS_CUDA(cudaStreamSynchronize(ctx->stream));
            ctx->dems.insert(dem);
        } catch (...) {
            if (dem->level0) tracked_free(dem->level0);
            if (dem->cells) tracked_free(dem->cells);
            if (dem->bounds) tracked_free(dem->bounds);
            delete dem;
            throw;
        }
        *out = dem;
    });
}

ls200_status ls200_dem_destroy(ls200_dem *dem) {
    return guard([&] {
        if (!dem) return;
        std::lock_guard<std::mutex> hold(dem->ctx->lock);
        activate(dem->ctx);
        cudaStreamSynchronize(dem->ctx->stream);
        dem->ctx->dems.erase(dem);
        if (dem->level0) tracked_free(dem->level0);
        if (dem->cells) tracked_free(dem->cells);
        if (dem->bounds) tracked_free(dem->bounds);
        delete dem;
    });
}

ls200_status ls200_dem_download_mips(ls200_dem *dem, float *mips, int64_t capacity) {
    return guard([&] {
        LS_REQUIRE(dem && mips, "NULL argument");
        LS_REQUIRE(capacity >= dem->mip_count, "mip buffer is too small");
        std::lock_guard<std::mutex> hold(dem->ctx->lock);
        activate(dem->ctx);
        if (dem->mip_count > 0)
            LS_CUDA(cudaMemcpyAsync(mips, dem->mips, sizeof(float) * dem->mip_count,
                                    cudaMemcpyDeviceToHost, dem->ctx->stream));
        LS_CUDA(cudaStreamSynchronize(dem->ctx->stream));
    });
}

ls200_status ls200_build_max_pyramid(ls200_context *ctx, const float *level0, int width,
                                     int height, float *mips) {
    ls200_dem *dem = nullptr;
    static const double zero6[6] = {0, 0, 0, 0, 0, 0};
    static const float zero11[11] = {0};
    ls200_status s =
        ls200_dem_create(ctx, level0, width, height, nullptr, zero6, zero6, zero11, &dem);
    if (s != LS200_OK) return s;
    s = ls200_dem_download_mips(dem, mips, dem->mip_count);
    ls200_status t = ls200_dem_destroy(dem);
    return s != LS200_OK ? s : t;
}

ls200_status ls200_dem_set_heights_device(ls200_dem *dem, const float *device_heights) {
    return guard([&] {
        LS_REQUIRE(dem && device_heights, "NULL argument");
        ls200_context *ctx = dem->ctx;
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LS_CUDA(cudaMemcpyAsync(dem->level0, device_heights,
                                sizeof(float) * size_t(dem->width) * dem->height,
                                cudaMemcpyDeviceToDevice, ctx->stream));
        build_pyramid_device(ctx, dem);
        sanitize_level0(ctx, dem);
        build_cell_bounds(ctx, dem);
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_dem_level0_device(ls200_dem *dem, const float **device_level0) {
    return guard([&] {
        LS_REQUIRE(dem && device_level0, "NULL argument");
        *device_level0 = dem->level0;
    });
}

ls200_status ls200_set_counting(ls200_context *ctx, int enabled) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        std::lock_guard<std::mutex> hold(ctx->lock);
        ctx->counting = enabled != 0;
    });
}

ls200_status ls200_last_counters(ls200_context *ctx, int64_t *visits, int64_t *samples,
                                 int64_t *steps) {
    return guard([&] {
        LS_REQUIRE(ctx != nullptr, "context is NULL");
        std::lock_guard<std::mutex> hold(ctx->lock);
        if (visits) *visits = static_cast<int64_t>(ctx->last_visits);
        if (samples) *samples = static_cast<int64_t>(ctx->last_samples);
        if (steps) *steps = static_cast<int64_t>(ctx->last_steps);
    });
}

}  // extern "C"
