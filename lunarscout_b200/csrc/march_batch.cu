// Persistent multi-site horizon march: every tile of a batch (tiles of many
// sites, DEMs of different sizes and resolutions, rays of very different
// lengths) in ONE launch.  One resident grid (SMs x occupancy) of 128-thread
// blocks; each warp takes the next 32-ray job from a global counter (work
// stealing), so long rays of one site never leave the GPU idle while a
// per-tile launch drains.  A thread marches its ray through all DEM passes
// with the slope carried in a register, and writes the pixel-major result
// (optionally degrees) directly: no per-pass launch, no working buffer, no
// transpose.
//
// Traversal 0 is the reference traversal (march_core.cuh), bit-identical to
// the per-tile kernel.  Traversal 1 adds the skip ladder (ladder_advance):
// a cull climbs to the largest culled ancestor cell, which removes most of
// the footprint-limited steps of long rays; its results are checked against
// its own CPU restatement (oracle flag OPT_LADDER) and their distance from
// the FP64 restatement is measured beside the reference traversal's.
//
// Launch configuration (autotuned, never changing results): how the 32 lanes
// of a job map onto rays (L adjacent pixels x 32/L adjacent azimuths, L a
// power of two up to 32), and the resident blocks per SM (8 at 64 registers,
// 6 at 80).
#include "march_core.cuh"

#include <map>
#include <vector>

namespace ls200 {

constexpr int kMaxSiteDems = 8;
constexpr int kTileSide = 128;
constexpr int kTilePixels = kTileSide * kTileSide;

// Host-built description of one DEM; the level table is derived on the
// device so that its float32 products round exactly as in the per-tile path.
struct BatchDemSource {
    const float *cells;
    const float *bounds;
    int width, height, level_count;
    int4 levels[kMaxLevels];
    float m6, m7, m9, m10, radius;
};

struct BatchDem {
    DemView view;
    LevelTable table;
};

struct BatchTile {
    const float *segments;  // [A, C, D, 18]
    float *out;             // [16384, A] pixel-major
    int dems[kMaxSiteDems];  // batch DEM indices, primary first
    int dem_count;
    int tile_column, tile_row;
    float observer_elevation;
};

struct SitesParams {
    const BatchDem *dems;
    const BatchTile *tiles;
    int azimuth_count, center_count, subpatch, degrees;
    int lanes_per_azimuth;  // 1..32 (power of two): pixels of one azimuth in a job
    long long pixel_groups, jobs_per_tile, job_count;
    unsigned long long *next_job;
    unsigned long long *counters;
    // Adjoint checkpoints (NULL when not recorded), per ray like `out`:
    // (px, py, true_m, slope) of the winning level-0 sample, and
    // flags = pass << 1 | near (0xff when no sample won).
    float4 *checkpoints;
    uint8_t *checkpoint_flags;
};

// Level table read through the read-only path (each warp may be on a
// different DEM; the tables stay resident in L1).
struct GlobalLevels {
    const LevelTable *t;
    __device__ __forceinline__ float side(int l) const { return __ldg(&t->side[l]); }
    __device__ __forceinline__ float fallback(int l) const { return __ldg(&t->fallback[l]); }
    __device__ __forceinline__ float out_step(int l) const { return __ldg(&t->out_step[l]); }
    __device__ __forceinline__ int4 cells(int l) const { return __ldg(&t->cells[l]); }
};

__global__ void batch_dem_kernel(const BatchDemSource *__restrict__ sources,
                                 BatchDem *__restrict__ dems) {
    const BatchDemSource &s = sources[blockIdx.x];
    BatchDem &d = dems[blockIdx.x];
    const float resolution = mean_resolution(s.m6, s.m7, s.m9, s.m10);
    if (threadIdx.x == 0)
        d.view = DemView{s.cells, s.bounds, s.width, s.height, s.level_count, resolution,
                         hypot_fused(s.m6, s.m9), s.radius};
    if (threadIdx.x < s.level_count)
        fill_level(d.table, threadIdx.x, resolution, s.levels[threadIdx.x]);
}

template <bool kArgmax>
struct TrackerOf {
    using type = NoArgmax;
};
template <>
struct TrackerOf<true> {
    using type = Argmax;
};

template <bool kCount, int kLadder, int kMinBlocks, bool kArgmax = false>
__global__ void __launch_bounds__(128, kMinBlocks)
    march_sites_kernel(const __grid_constant__ SitesParams P) {
    const int lane = threadIdx.x & 31;
    const int lanes = P.lanes_per_azimuth;
    const int azimuths_per_job = 32 / lanes;
    unsigned visits = 0, samples = 0, steps = 0;
    for (;;) {
        unsigned long long taken = 0;
        if (lane == 0) taken = atomicAdd(P.next_job, 1ull);
        const long long job = static_cast<long long>(__shfl_sync(0xffffffffu, taken, 0));
        if (job >= P.job_count) break;
        const int t = static_cast<int>(job / P.jobs_per_tile);
        const long long local = job - t * P.jobs_per_tile;
        const int azimuth_group = static_cast<int>(local / P.pixel_groups);
        const int pixel_group = static_cast<int>(local - azimuth_group * P.pixel_groups);
        const int pixel = pixel_group * lanes + lane % lanes;
        const int azimuth = azimuth_group * azimuths_per_job + lane / lanes;
        if (azimuth >= P.azimuth_count) continue;
        const BatchTile &tile = P.tiles[t];
        const int row = pixel / kTileSide, column = pixel % kTileSide;
        const size_t ray = static_cast<size_t>(pixel) * P.azimuth_count + azimuth;
        float *out = tile.out + ray;
        const BatchDem &primary = P.dems[tile.dems[0]];
        const int primary_width = primary.view.width, primary_height = primary.view.height;
        typename TrackerOf<kArgmax>::type tracker;
        const size_t checkpoint = static_cast<size_t>(t) * kTilePixels * P.azimuth_count + ray;
        // Pixels outside the primary DEM keep the -inf sentinel.
        if (tile.tile_column + column >= primary_width || tile.tile_row + row >= primary_height) {
            *out = -INFINITY;
            if (kArgmax) P.checkpoint_flags[checkpoint] = 0xff;
            continue;
        }
        const float observer_z = __fadd_rn(
            bilinear(primary.view.cells, primary_width, primary_height,
                     static_cast<float>(tile.tile_column + column),
                     static_cast<float>(tile.tile_row + row)),
            tile.observer_elevation);
        float current = -1e30f;
        for (int d = 0; d < tile.dem_count; ++d) {
            const BatchDem &dem = P.dems[tile.dems[d]];
            const DemView view = dem.view;
            const float ratio = __fdiv_rn(primary.view.column_res, view.column_res);
            const RaySegment g = interpolate_segment<(kLadder & kRelative) != 0>(
                tile.segments, P.center_count, tile.dem_count, d, azimuth, column, row,
                tile.tile_column, tile.tile_row, kTileSide, P.subpatch, primary_width,
                primary_height, ratio);
            if constexpr (kArgmax) tracker.current_pass = d;
            current = march_dem_tracked<kCount, kLadder>(GlobalLevels{&dem.table}, view, g, d,
                                                         observer_z, current, visits, samples,
                                                         steps, tracker);
        }
        if constexpr (kArgmax) {
            P.checkpoints[checkpoint] =
                make_float4(tracker.px, tracker.py, tracker.true_m, tracker.slope);
            P.checkpoint_flags[checkpoint] =
                tracker.pass < 0 ? uint8_t(0xff)
                                 : static_cast<uint8_t>((tracker.pass << 1) | tracker.near);
        }
        float value = current > -1e29f ? current : -INFINITY;
        if (P.degrees && !isinf(value)) value = __fmul_rn(atanf(value), kSlopeDegrees);
        *out = value;
    }
    if (kCount) add_counters(P.counters, visits, samples, steps);
}

template <bool kCount, int kLadder, int kMinBlocks, bool kArgmax = false>
static void launch_sites(ls200_context *ctx, const SitesParams &P) {
    int per_sm = 0;
    LS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, march_sites_kernel<kCount, kLadder, kMinBlocks, kArgmax>, 128, 0));
    const int blocks = ctx->props.multiProcessorCount * (per_sm > 0 ? per_sm : 1);
    march_sites_kernel<kCount, kLadder, kMinBlocks, kArgmax><<<blocks, 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
}

template <bool kCount, int kMinBlocks>
static void dispatch(ls200_context *ctx, const SitesParams &P, int traversal) {
    switch (traversal) {
        case kReference: launch_sites<kCount, kReference, kMinBlocks>(ctx, P); break;
        case kLadderClimb: launch_sites<kCount, kLadderClimb, kMinBlocks>(ctx, P); break;
        case kRelative: launch_sites<kCount, kRelative, kMinBlocks>(ctx, P); break;
        default: launch_sites<kCount, kLadderClimb | kRelative, kMinBlocks>(ctx, P); break;
    }
}

// The checkpointing march runs 8 blocks per SM too: its extra tracker
// registers spill a little at 64, which costs less than the occupancy of 6
// blocks at 80 registers (measured: the differentiable workload's forward
// 294 -> 267 ms, the 8192^2 slice's 2.58 -> 2.04 s).
static void dispatch_argmax(ls200_context *ctx, const SitesParams &P, int traversal) {
    if (traversal == kReference) launch_sites<false, kReference, 8, true>(ctx, P);
    else launch_sites<false, kLadderClimb, 8, true>(ctx, P);
}

static size_t align_up(size_t n) { return (n + 255) & ~size_t(255); }

void march_sites_run(ls200_context *ctx, const ls200_site_tile *tiles, int tile_count,
                     int azimuth_count, int subpatch_size, int traversal, bool degrees,
                     float *device_out, double *seconds, float4 *checkpoints,
                     uint8_t *checkpoint_flags) {
    {
        LS_REQUIRE(ctx && tiles && device_out, "NULL argument");
        LS_REQUIRE(tile_count > 0, "tile_count must be positive");
        LS_REQUIRE(traversal >= 0 && traversal <= (kLadderClimb | kRelative),
                   "traversal must be 0 to 3");
        LS_REQUIRE(azimuth_count > 0 && static_cast<int64_t>(kTilePixels) * azimuth_count <
                                            (int64_t(1) << 31),
                   "azimuth_count is out of range");
        LS_REQUIRE(subpatch_size == 2 || subpatch_size == 4 || subpatch_size == 8 ||
                       subpatch_size == 16 || subpatch_size == 32 || subpatch_size == 64 ||
                       subpatch_size == 128,
                   "subpatch_size must be a power of two between 2 and 128");
        const int count = kTileSide / subpatch_size + 2;
        const int center_count = count * count;
        std::map<const ls200_dem *, int> index;
        std::vector<ls200_dem *> unique;
        size_t segment_floats = 0;
        for (int t = 0; t < tile_count; ++t) {
            const ls200_site_tile &tile = tiles[t];
            LS_REQUIRE(tile.dems && tile.dem_count > 0 && tile.dem_count <= kMaxSiteDems,
                       "each tile needs 1 to 8 DEMs");
            for (int d = 0; d < tile.dem_count; ++d) {
                ls200_dem *dem = tile.dems[d];
                LS_REQUIRE(dem != nullptr, "NULL DEM");
                LS_REQUIRE(dem->ctx == ctx, "DEM belongs to another context");
                LS_REQUIRE(dem->width >= 2 && dem->height >= 2, "DEMs must be at least 2x2 pixels");
                if (!index.count(dem)) {
                    index[dem] = static_cast<int>(unique.size());
                    unique.push_back(dem);
                }
            }
            const ls200_dem *primary = tile.dems[0];
            LS_REQUIRE(tile.tile_column >= 0 && tile.tile_row >= 0 &&
                           tile.tile_column < primary->width && tile.tile_row < primary->height,
                       "tile origin lies outside the primary DEM");
            LS_REQUIRE(tile.maximum_distance_m > 0.0, "maximum_distance_m must be positive");
            segment_floats += static_cast<size_t>(azimuth_count) * center_count * tile.dem_count *
                              kSegmentFields;
        }
        std::unique_lock<std::mutex> hold(ctx->lock);
        activate(ctx);
        ctx->segments.reserve(segment_floats * sizeof(float));
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[0], ctx->stream));
        std::vector<BatchTile> host_tiles(tile_count);
        float *segments = ctx->segments.as<float>();
        float *out = static_cast<float *>(device_out);
        for (int t = 0; t < tile_count; ++t) {
            const ls200_site_tile &tile = tiles[t];
            segments_device(ctx, tile.dems, tile.dem_count, tile.tile_column, tile.tile_row,
                            kTileSide, azimuth_count, tile.maximum_distance_m,
                            tile.observer_elevation_m, subpatch_size, segments);
            BatchTile &bt = host_tiles[t];
            bt.segments = segments;
            bt.out = out + static_cast<size_t>(t) * kTilePixels * azimuth_count;
            for (int d = 0; d < kMaxSiteDems; ++d)
                bt.dems[d] = d < tile.dem_count ? index[tile.dems[d]] : 0;
            bt.dem_count = tile.dem_count;
            bt.tile_column = tile.tile_column;
            bt.tile_row = tile.tile_row;
            bt.observer_elevation = tile.observer_elevation_m;
            segments += static_cast<size_t>(azimuth_count) * center_count * tile.dem_count *
                        kSegmentFields;
        }
        // The batch tables go to the context scratch only now: segment
        // generation above uses (and may grow) the same buffer.
        const size_t dem_count = unique.size();
        const size_t off_sources = 0;
        const size_t off_dems = align_up(off_sources + dem_count * sizeof(BatchDemSource));
        const size_t off_tiles = align_up(off_dems + dem_count * sizeof(BatchDem));
        const size_t off_job = align_up(off_tiles + tile_count * sizeof(BatchTile));
        ctx->scratch.reserve(off_job + sizeof(unsigned long long));
        char *scratch = ctx->scratch.as<char>();
        std::vector<BatchDemSource> sources(dem_count);
        for (size_t i = 0; i < dem_count; ++i) {
            const ls200_dem *dem = unique[i];
            BatchDemSource &s = sources[i];
            s.cells = dem->cells;
            s.bounds = dem->bounds;
            s.width = dem->width;
            s.height = dem->height;
            s.level_count = dem->level_count;
            const int cells0 = dem->width * dem->height;
            for (int l = 0; l < kMaxLevels; ++l)
                s.levels[l] = l < dem->level_count
                                  ? make_int4(l == 0 ? 0 : cells0 + dem->levels[l].offset,
                                              dem->levels[l].width, dem->levels[l].height, 0)
                                  : make_int4(0, 0, 0, 0);
            s.m6 = dem->map_parameters[6];
            s.m7 = dem->map_parameters[7];
            s.m9 = dem->map_parameters[9];
            s.m10 = dem->map_parameters[10];
            s.radius = static_cast<float>(dem->projection[0]);
        }
        LS_CUDA(cudaMemcpyAsync(scratch + off_sources, sources.data(),
                                dem_count * sizeof(BatchDemSource), cudaMemcpyHostToDevice,
                                ctx->stream));
        LS_CUDA(cudaMemcpyAsync(scratch + off_tiles, host_tiles.data(),
                                tile_count * sizeof(BatchTile), cudaMemcpyHostToDevice,
                                ctx->stream));
        LS_CUDA(cudaMemsetAsync(scratch + off_job, 0, sizeof(unsigned long long), ctx->stream));
        batch_dem_kernel<<<static_cast<unsigned>(dem_count), 32, 0, ctx->stream>>>(
            reinterpret_cast<const BatchDemSource *>(scratch + off_sources),
            reinterpret_cast<BatchDem *>(scratch + off_dems));
        LS_CUDA(cudaGetLastError());
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[1], ctx->stream));

        SitesParams P{};
        P.dems = reinterpret_cast<const BatchDem *>(scratch + off_dems);
        P.tiles = reinterpret_cast<const BatchTile *>(scratch + off_tiles);
        P.azimuth_count = azimuth_count;
        P.center_count = center_count;
        P.subpatch = subpatch_size;
        P.degrees = degrees ? 1 : 0;
        P.lanes_per_azimuth = ctx->batch_lanes_per_azimuth;
        const int azimuths_per_job = 32 / P.lanes_per_azimuth;
        P.pixel_groups = kTilePixels / P.lanes_per_azimuth;
        P.jobs_per_tile = P.pixel_groups * ((azimuth_count + azimuths_per_job - 1) /
                                            azimuths_per_job);
        P.job_count = P.jobs_per_tile * tile_count;
        P.next_job = reinterpret_cast<unsigned long long *>(scratch + off_job);
        P.counters = ctx->counters.as<unsigned long long>();
        P.checkpoints = checkpoints;
        P.checkpoint_flags = checkpoint_flags;
        reset_counters(ctx);
        if (checkpoints) dispatch_argmax(ctx, P, traversal);
        else if (ctx->counting) dispatch<true, 8>(ctx, P, traversal);
        else if (ctx->batch_min_blocks == 6) dispatch<false, 6>(ctx, P, traversal);
        else dispatch<false, 8>(ctx, P, traversal);
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[2], ctx->stream));
        // The host tables above must outlive their copies.
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (seconds) {
            float ms = 0.0f;
            LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
            seconds[0] = ms / 1000.0;
            LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[1], ctx->events[2]));
            seconds[1] = ms / 1000.0;
        }
        resolve_counters(ctx);
    }
}

}  // namespace ls200

using namespace ls200;

extern "C" ls200_status ls200_march_sites(ls200_context *ctx, const ls200_site_tile *tiles,
                                          int tile_count, int azimuth_count, int subpatch_size,
                                          int traversal, int degrees, void *device_out,
                                          double *seconds) {
    return guard([&] {
        march_sites_run(ctx, tiles, tile_count, azimuth_count, subpatch_size, traversal,
                        degrees != 0, static_cast<float *>(device_out), seconds, nullptr,
                        nullptr);
    });
}

extern "C" ls200_status ls200_set_batch_config(ls200_context *ctx, int lanes_per_azimuth,
                                               int min_blocks) {
    return guard([&] {
        LS_REQUIRE(ctx, "NULL argument");
        LS_REQUIRE(lanes_per_azimuth >= 1 && lanes_per_azimuth <= 32 &&
                       (lanes_per_azimuth & (lanes_per_azimuth - 1)) == 0,
                   "lanes_per_azimuth must be a power of two from 1 to 32");
        LS_REQUIRE(min_blocks == 6 || min_blocks == 8, "min_blocks must be 6 or 8");
        std::lock_guard<std::mutex> hold(ctx->lock);
        ctx->batch_lanes_per_azimuth = lanes_per_azimuth;
        ctx->batch_min_blocks = min_blocks;
    });
}

extern "C" ls200_status ls200_get_batch_config(ls200_context *ctx, int *lanes_per_azimuth,
                                               int *min_blocks) {
    return guard([&] {
        LS_REQUIRE(ctx && lanes_per_azimuth && min_blocks, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        *lanes_per_azimuth = ctx->batch_lanes_per_azimuth;
        *min_blocks = ctx->batch_min_blocks;
    });
}
