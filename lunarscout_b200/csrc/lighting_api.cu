// C-ABI entry points of the lighting products.
#include "lighting.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace ls200 {

struct LightingState {
    DeviceBuffer dem, horizons, frames, out;
    DeviceBuffer duration_frames, duration_bits, duration_tables;  // mission duration
    DeviceBuffer haven_bits, haven_months, haven_longest, haven_flags;  // safe haven
    DeviceBuffer visibility;  // Earth visibility: counts, then the valid table
    TileGeo geo{};
    bool loaded = false;
    std::set<ls200_vectors *> vectors;  // live vector tables of the context
};

static LightingState &state_of(ls200_context *ctx) {
    if (!ctx->lighting) ctx->lighting = new LightingState();
    return *ctx->lighting;
}

void release_lighting_state(ls200_context *ctx) {
    if (!ctx->lighting) return;
    for (ls200_vectors *v : ctx->lighting->vectors) {
        tracked_free(v->data);
        tracked_free(v->order);
        tracked_free(v->window);
        delete v;
    }
    delete ctx->lighting;
    ctx->lighting = nullptr;
}

static void check_valid(int valid_width, int valid_height) {
    LS_REQUIRE(valid_width >= 1 && valid_width <= kPatch && valid_height >= 1 &&
                   valid_height <= kPatch,
               "valid patch dimensions must be between 1 and 128");
}

static LightingBatch single_batch(LightingState &st, const ls200_vectors *v) {
    LightingBatch B{};
    B.tiles[0] = st.geo;
    B.patch_dem = st.dem.as<float>();
    B.horizons = st.horizons.as<float>();
    B.vectors = v ? v->data : nullptr;
    B.frames = st.frames.as<float>();
    return B;
}

}  // namespace ls200

using namespace ls200;

extern "C" {

ls200_status ls200_vectors_create(ls200_context *ctx, const float *vectors, int count,
                                  ls200_vectors **out) {
    return guard([&] {
        LS_REQUIRE(ctx && vectors && out, "NULL argument");
        LS_REQUIRE(count > 0, "at least one vector is required");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        // Time indices by longitude (ties by index); non-finite keys sort as 0.
        std::vector<double> key(count);
        for (int t = 0; t < count; ++t) {
            const double k = std::atan2(static_cast<double>(vectors[3 * t + 1]),
                                        static_cast<double>(vectors[3 * t]));
            key[t] = std::isfinite(k) ? k : 0.0;
        }
        std::vector<int> order(count);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return key[a] < key[b]; });
        auto v = new ls200_vectors();
        v->ctx = ctx;
        v->count = count;
        auto release = [&] {
            if (v->data) tracked_free(v->data);
            if (v->order) tracked_free(v->order);
            if (v->window) tracked_free(v->window);
            delete v;
        };
        cudaError_t e = tracked_malloc(&v->data, sizeof(float) * 3 * size_t(count));
        if (e == cudaSuccess) e = tracked_malloc(&v->order, sizeof(int) * size_t(count));
        if (e == cudaSuccess) e = tracked_malloc(&v->window, sizeof(int) * size_t(count));
        if (e != cudaSuccess) {
            release();
            throw Error(LS200_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        e = cudaMemcpyAsync(v->data, vectors, sizeof(float) * 3 * size_t(count),
                            cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(v->order, order.data(), sizeof(int) * size_t(count),
                                cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            release();
            throw Error(LS200_ERR_CUDA, std::string("vector upload: ") + cudaGetErrorString(e));
        }
        state_of(ctx).vectors.insert(v);
        *out = v;
    });
}

ls200_status ls200_vectors_destroy(ls200_vectors *vectors) {
    return guard([&] {
        if (!vectors) return;
        std::lock_guard<std::mutex> hold(vectors->ctx->lock);
        activate(vectors->ctx);
        cudaStreamSynchronize(vectors->ctx->stream);
        state_of(vectors->ctx).vectors.erase(vectors);
        tracked_free(vectors->data);
        tracked_free(vectors->order);
        tracked_free(vectors->window);
        delete vectors;
    });
}

ls200_status ls200_lighting_load(ls200_context *ctx, const float *patch_dem,
                                 const double *geo_transform, const double *projection,
                                 const float *horizons, int tile_x, int tile_y,
                                 int valid_width, int valid_height) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dem && geo_transform && projection && horizons, "NULL argument");
        check_valid(valid_width, valid_height);
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        const size_t plane = size_t(kPatch) * kPatch;
        st.dem.reserve(sizeof(float) * plane);
        st.horizons.reserve(sizeof(float) * plane * kAzimuths);
        st.frames.reserve(sizeof(float) * plane * 12);
        LS_CUDA(cudaMemcpyAsync(st.dem.ptr, patch_dem, sizeof(float) * plane,
                                cudaMemcpyHostToDevice, ctx->stream));
        LS_CUDA(cudaMemcpyAsync(st.horizons.ptr, horizons, sizeof(float) * plane * kAzimuths,
                                cudaMemcpyHostToDevice, ctx->stream));
        std::memcpy(st.geo.gt, geo_transform, sizeof st.geo.gt);
        std::memcpy(st.geo.proj, projection, sizeof st.geo.proj);
        st.geo.tile_x = tile_x;
        st.geo.tile_y = tile_y;
        st.geo.valid_width = valid_width;
        st.geo.valid_height = valid_height;
        st.loaded = true;
    });
}

ls200_status ls200_lighting_run(ls200_context *ctx, const ls200_vectors *vectors,
                                int time_start, int time_count, int signal, void *out) {
    return guard([&] {
        LS_REQUIRE(ctx && vectors && out, "NULL argument");
        LS_REQUIRE(signal >= kSignalFraction && signal <= kSignalMargin, "unknown signal");
        LS_REQUIRE(time_start >= 0 && time_count > 0 &&
                       int64_t(time_start) + time_count <= int64_t(vectors->count),
                   "time range outside the vector table");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        LS_REQUIRE(st.loaded, "no lighting tile is loaded");
        const size_t plane = size_t(kPatch) * kPatch;
        const size_t item = signal == kSignalBytes ? 1 : sizeof(float);
        const size_t bytes = item * plane * size_t(time_count);
        st.out.reserve(bytes);
        LightingBatch B = single_batch(st, vectors);
        B.out = st.out.ptr;
        B.time_start = time_start;
        B.time_count = time_count;
        lighting_launch(ctx, B, 1, signal);
        LS_CUDA(cudaMemcpyAsync(out, st.out.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_psr_run(ls200_context *ctx, const ls200_vectors *vectors, uint8_t *out) {
    return guard([&] {
        LS_REQUIRE(ctx && vectors && out, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        LS_REQUIRE(st.loaded, "no lighting tile is loaded");
        const size_t plane = size_t(kPatch) * kPatch;
        st.out.reserve(plane);
        LightingBatch B = single_batch(st, vectors);
        B.out = st.out.ptr;
        B.time_start = 0;
        B.time_count = vectors->count;
        lighting_launch(ctx, B, 1, kSignalPsr);
        LS_CUDA(cudaMemcpyAsync(out, st.out.ptr, plane, cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_lighting_device(ls200_context *ctx, int tile_count, const float *patch_dems,
                                   const double *geo_transforms, const double *projections,
                                   const int32_t *windows, const float *horizons,
                                   const ls200_vectors *vectors, int time_start,
                                   int time_count, int signal, float *frames, void *out) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dems && geo_transforms && projections && windows && horizons &&
                       vectors && frames && out,
                   "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kMaxBatchTiles,
                   "tile_count must be between 1 and 32");
        LS_REQUIRE(signal >= kSignalFraction && signal <= kSignalPsr, "unknown signal");
        LS_REQUIRE(time_start >= 0 && time_count > 0 &&
                       int64_t(time_start) + time_count <= int64_t(vectors->count),
                   "time range outside the vector table");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingBatch B{};
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, geo_transforms + 6 * t, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, projections + 6 * t, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = windows[4 * t + 0];
            B.tiles[t].tile_y = windows[4 * t + 1];
            B.tiles[t].valid_width = windows[4 * t + 2];
            B.tiles[t].valid_height = windows[4 * t + 3];
            check_valid(B.tiles[t].valid_width, B.tiles[t].valid_height);
        }
        B.patch_dem = patch_dems;
        B.horizons = horizons;
        B.vectors = vectors->data;
        B.frames = frames;
        B.out = out;
        B.time_start = signal == kSignalPsr ? 0 : time_start;
        B.time_count = signal == kSignalPsr ? vectors->count : time_count;
        lighting_launch(ctx, B, tile_count, signal, vectors);
    });
}

ls200_status ls200_mission_duration_device(
    ls200_context *ctx, int tile_count, const float *patch_dems, const double *geo_transforms,
    const double *projections, const int32_t *windows, const float *horizons,
    const ls200_vectors *sun, const ls200_vectors *earth, float sun_threshold,
    float earth_threshold, const double *sample_hours, const int32_t *start_windows,
    int interval_count, int output_days, float *out) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dems && geo_transforms && projections && windows && horizons &&
                       sun && sample_hours && start_windows && out,
                   "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kMaxBatchTiles,
                   "tile_count must be between 1 and 32");
        LS_REQUIRE(interval_count >= 1 && interval_count <= 64,
                   "interval_count must be between 1 and 64");
        LS_REQUIRE(sun->ctx == ctx && sun->count > 0, "sun vectors belong to another context");
        LS_REQUIRE(!earth || (earth->ctx == ctx && earth->count == sun->count),
                   "earth vectors must match the sun vectors' time axis");
        const int count = sun->count;
        std::vector<int2> intervals(interval_count);
        for (int i = 0; i < interval_count; ++i) {
            intervals[i] = make_int2(start_windows[2 * i], start_windows[2 * i + 1]);
            LS_REQUIRE(intervals[i].x >= 0 && intervals[i].x <= intervals[i].y &&
                           intervals[i].y <= count,
                       "start windows must be sample index ranges within the time axis");
        }
        bool integral = true;
        double total = 0.0;
        for (int t = 0; t < count; ++t) {
            LS_REQUIRE(std::isfinite(sample_hours[t]) && sample_hours[t] >= 0.0,
                       "sample durations must be finite and non-negative");
            integral = integral && sample_hours[t] == std::floor(sample_hours[t]);
            total += sample_hours[t];
        }
        integral = integral && total < 9.0e15;
        std::vector<double> prefix;
        if (integral) {
            prefix.resize(count + 1);
            prefix[0] = 0.0;
            for (int t = 0; t < count; ++t) prefix[t + 1] = prefix[t] + sample_hours[t];
        }
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        LightingBatch B{};
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, geo_transforms + 6 * t, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, projections + 6 * t, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = windows[4 * t + 0];
            B.tiles[t].tile_y = windows[4 * t + 1];
            B.tiles[t].valid_width = windows[4 * t + 2];
            B.tiles[t].valid_height = windows[4 * t + 3];
            check_valid(B.tiles[t].valid_width, B.tiles[t].valid_height);
        }
        const size_t plane = static_cast<size_t>(kPatch) * kPatch;
        const size_t words = (static_cast<size_t>(count) + 31) / 32;
        const size_t frames_bytes = sizeof(float) * 12 * tile_count * plane;
        // One bit stream for the Sun's condition, a second for the Earth's.
        const size_t bits_bytes = sizeof(uint32_t) * tile_count * plane * words * (earth ? 2 : 1);
        const size_t table_bytes = sizeof(double) * (2 * size_t(count) + 1) +
                                   sizeof(int2) * interval_count;
        st.duration_frames.reserve(frames_bytes);
        st.duration_bits.reserve(bits_bytes);
        st.duration_tables.reserve(table_bytes);
        double *d_hours = st.duration_tables.as<double>();
        double *d_prefix = d_hours + count;
        int2 *d_windows = reinterpret_cast<int2 *>(d_prefix + count + 1);
        LS_CUDA(cudaMemcpyAsync(d_hours, sample_hours, sizeof(double) * count,
                                cudaMemcpyHostToDevice, ctx->stream));
        if (integral)
            LS_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(double) * (count + 1),
                                    cudaMemcpyHostToDevice, ctx->stream));
        LS_CUDA(cudaMemcpyAsync(d_windows, intervals.data(), sizeof(int2) * interval_count,
                                cudaMemcpyHostToDevice, ctx->stream));
        B.patch_dem = patch_dems;
        B.horizons = horizons;
        B.vectors = sun->data;
        B.frames = st.duration_frames.as<float>();
        B.time_start = 0;
        B.time_count = count;
        mission_duration_launch(ctx, B, tile_count, earth ? earth->data : nullptr,
                                sun_threshold, earth_threshold, st.duration_bits.as<uint32_t>(),
                                d_hours, integral ? d_prefix : nullptr, d_windows,
                                interval_count, output_days != 0, out, sun->order,
                                earth ? earth->order : nullptr);
        // The host tables above must outlive their copies.
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_safe_haven_device(
    ls200_context *ctx, int tile_count, const float *patch_dems, const double *geo_transforms,
    const double *projections, const int32_t *windows, const float *horizons,
    const ls200_vectors *sun, const ls200_vectors *earth, float sunlight_threshold,
    float earth_threshold_deg, float time_step_hours, const int32_t *month_index_of,
    int band_count, float *out) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dems && geo_transforms && projections && windows && horizons &&
                       sun && earth && month_index_of && out,
                   "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kMaxBatchTiles,
                   "tile_count must be between 1 and 32");
        LS_REQUIRE(sun->ctx == ctx && earth->ctx == ctx && sun->count > 0,
                   "vectors belong to another context");
        LS_REQUIRE(earth->count == sun->count,
                   "earth vectors must match the sun vectors' time axis");
        LS_REQUIRE(sunlight_threshold >= 0.0f && sunlight_threshold <= 1.0f,
                   "sunlight_threshold must be between zero and one");
        LS_REQUIRE(std::isfinite(earth_threshold_deg), "earth_threshold_deg must be finite");
        LS_REQUIRE(std::isfinite(time_step_hours) && time_step_hours > 0.0f,
                   "time_step_hours must be positive and finite");
        LS_REQUIRE(band_count >= 1 && band_count <= 65536,
                   "band_count must be between 1 and 65536");
        const int count = sun->count;
        for (int t = 0; t < count; ++t)
            LS_REQUIRE(month_index_of[t] >= -1 && month_index_of[t] < band_count,
                       "month indices must be -1 or a band index");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        LightingBatch B{};
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, geo_transforms + 6 * t, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, projections + 6 * t, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = windows[4 * t + 0];
            B.tiles[t].tile_y = windows[4 * t + 1];
            B.tiles[t].valid_width = windows[4 * t + 2];
            B.tiles[t].valid_height = windows[4 * t + 3];
            check_valid(B.tiles[t].valid_width, B.tiles[t].valid_height);
        }
        const size_t plane = static_cast<size_t>(kPatch) * kPatch;
        const size_t words = (static_cast<size_t>(count) + 31) / 32;
        const size_t cells = static_cast<size_t>(tile_count) * band_count * plane;
        st.duration_frames.reserve(sizeof(float) * 12 * tile_count * plane);
        st.haven_bits.reserve(sizeof(uint32_t) * 2 * tile_count * words * plane);
        st.haven_months.reserve(sizeof(int32_t) * count);
        st.haven_longest.reserve(sizeof(int32_t) * cells);
        st.haven_flags.reserve(cells);
        LS_CUDA(cudaMemcpyAsync(st.haven_months.as<int32_t>(), month_index_of,
                                sizeof(int32_t) * count, cudaMemcpyHostToDevice, ctx->stream));
        B.patch_dem = patch_dems;
        B.horizons = horizons;
        B.vectors = sun->data;
        B.frames = st.duration_frames.as<float>();
        B.time_start = 0;
        B.time_count = count;
        safe_haven_launch(ctx, B, tile_count, earth->data, sunlight_threshold,
                          earth_threshold_deg, st.haven_bits.as<uint32_t>(),
                          st.haven_months.as<int32_t>(), band_count, time_step_hours,
                          st.haven_longest.as<int32_t>(), st.haven_flags.as<uint8_t>(), out,
                          sun->order, earth->order);
        // The host month table must outlive its copy.
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_earth_visibility_device(ls200_context *ctx, int tile_count,
                                           const float *patch_dems,
                                           const double *geo_transforms,
                                           const double *projections, const int32_t *windows,
                                           const float *horizons, const ls200_vectors *earth,
                                           float threshold_deg, float *out) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dems && geo_transforms && projections && windows && horizons &&
                       earth && out,
                   "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kMaxBatchTiles,
                   "tile_count must be between 1 and 32");
        LS_REQUIRE(earth->ctx == ctx && earth->count > 0, "earth vectors belong to another context");
        LS_REQUIRE(std::isfinite(threshold_deg), "threshold_deg must be finite");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingState &st = state_of(ctx);
        LightingBatch B{};
        std::vector<int2> valid(tile_count);
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, geo_transforms + 6 * t, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, projections + 6 * t, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = windows[4 * t + 0];
            B.tiles[t].tile_y = windows[4 * t + 1];
            B.tiles[t].valid_width = windows[4 * t + 2];
            B.tiles[t].valid_height = windows[4 * t + 3];
            check_valid(B.tiles[t].valid_width, B.tiles[t].valid_height);
            valid[t] = make_int2(B.tiles[t].valid_width, B.tiles[t].valid_height);
        }
        const size_t plane = static_cast<size_t>(kPatch) * kPatch;
        const size_t counts_bytes = sizeof(unsigned) * tile_count * plane;
        st.duration_frames.reserve(sizeof(float) * 12 * tile_count * plane);
        st.visibility.reserve(counts_bytes + sizeof(int2) * kMaxBatchTiles);
        int2 *d_valid = reinterpret_cast<int2 *>(st.visibility.as<char>() + counts_bytes);
        LS_CUDA(cudaMemcpyAsync(d_valid, valid.data(), sizeof(int2) * tile_count,
                                cudaMemcpyHostToDevice, ctx->stream));
        B.patch_dem = patch_dems;
        B.horizons = horizons;
        B.vectors = earth->data;
        B.frames = st.duration_frames.as<float>();
        B.time_start = 0;
        B.time_count = earth->count;
        visibility_launch(ctx, B, tile_count, threshold_deg, st.visibility.as<unsigned>(),
                          d_valid, out, earth->order);
        // The host valid table must outlive its copy.
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

ls200_status ls200_sun_fraction(ls200_context *ctx, const float *horizons,
                                const float *azimuth_deg, const float *elevation_deg, int n,
                                float *out) {
    return guard([&] {
        LS_REQUIRE(ctx && horizons && azimuth_deg && elevation_deg && out && n > 0,
                   "invalid arguments");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        const size_t rows = sizeof(float) * size_t(n) * kAzimuths;
        ctx->scratch.reserve(rows + 3 * sizeof(float) * size_t(n));
        float *d_h = ctx->scratch.as<float>();
        float *d_a = d_h + size_t(n) * kAzimuths;
        float *d_e = d_a + n;
        float *d_o = d_e + n;
        LS_CUDA(cudaMemcpyAsync(d_h, horizons, rows, cudaMemcpyHostToDevice, ctx->stream));
        LS_CUDA(cudaMemcpyAsync(d_a, azimuth_deg, sizeof(float) * n, cudaMemcpyHostToDevice,
                                ctx->stream));
        LS_CUDA(cudaMemcpyAsync(d_e, elevation_deg, sizeof(float) * n, cudaMemcpyHostToDevice,
                                ctx->stream));
        sun_fraction_launch(ctx, d_h, d_a, d_e, n, d_o);
        LS_CUDA(cudaMemcpyAsync(out, d_o, sizeof(float) * n, cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of ls200_lighting_device.
//
// Some callers cannot call cudaMalloc at the point where they run the
// lighting products: a service whose device memory is owned by another
// allocator (a framework's caching allocator, a memory pool sized at start-up)
// may not take raw allocations, and a latency-bounded production loop cannot
// afford cudaMalloc/cudaFree, which may synchronise the whole device.  Those
// callers pass their own device inputs and outputs; the only working memory
// this kernel needs beyond them, the per-pixel frame table, lives in the
// fixed array below.
namespace ls200 {

// Scratch of the allocation-free entry point: per-pixel frames (12 floats for
// each of the 128x128 pixels) of up to kNoAllocTiles tiles = 3 MiB.  Every GPU
// that loads this library holds it until the process exits.
constexpr int kNoAllocTiles = 4;
static __device__ __align__(256) float g_noalloc_frames[size_t(kNoAllocTiles) * kPatch *
                                                        kPatch * 12];

static std::mutex g_noalloc_lock;
static float *g_noalloc_address[64] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the host-side symbol is only a stand-in for it).
static float *noalloc_frames(int device) {
    LS_REQUIRE(device >= 0 && device < 64, "device index out of range");
    std::lock_guard<std::mutex> hold(g_noalloc_lock);
    if (!g_noalloc_address[device]) {
        void *address = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&address, g_noalloc_frames);
        if (e != cudaSuccess || address == nullptr)
            throw Error(LS200_ERR_CUDA, std::string("cudaGetSymbolAddress(frame scratch): ") +
                                            cudaGetErrorString(e));
        g_noalloc_address[device] = static_cast<float *>(address);
    }
    return g_noalloc_address[device];
}

}  // namespace ls200

extern "C" {

ls200_status ls200_lighting_device_noalloc(ls200_context *ctx, int tile_count,
                                           const float *patch_dems,
                                           const double *geo_transforms,
                                           const double *projections, const int32_t *windows,
                                           const float *horizons, const float *device_vectors,
                                           int vector_count, int time_start, int time_count,
                                           int signal, void *out) {
    return guard([&] {
        LS_REQUIRE(ctx && patch_dems && geo_transforms && projections && windows && horizons &&
                       device_vectors && out,
                   "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kNoAllocTiles,
                   "the allocation-free lighting entry point takes 1 to 4 tiles per call "
                   "(its fixed frame scratch holds 4 tiles)");
        LS_REQUIRE(signal >= kSignalFraction && signal <= kSignalPsr, "unknown signal");
        LS_REQUIRE(vector_count > 0, "at least one vector is required");
        LS_REQUIRE(signal == kSignalPsr ||
                       (time_start >= 0 && time_count > 0 &&
                        int64_t(time_start) + int64_t(time_count) <= int64_t(vector_count)),
                   "time range outside the vector table");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        LightingBatch B{};
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, geo_transforms + 6 * t, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, projections + 6 * t, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = windows[4 * t + 0];
            B.tiles[t].tile_y = windows[4 * t + 1];
            B.tiles[t].valid_width = windows[4 * t + 2];
            B.tiles[t].valid_height = windows[4 * t + 3];
            check_valid(B.tiles[t].valid_width, B.tiles[t].valid_height);
        }
        B.patch_dem = patch_dems;
        B.horizons = horizons;
        B.vectors = device_vectors;
        // The frames kernel writes every entry it later reads (zeros outside
        // the valid window), so nothing in the scratch must start at zero.
        B.frames = noalloc_frames(ctx->device);
        B.out = out;
        B.time_start = signal == kSignalPsr ? 0 : time_start;
        B.time_count = signal == kSignalPsr ? vector_count : time_count;
        lighting_launch(ctx, B, tile_count, signal);
    });
}

}  // extern "C"
