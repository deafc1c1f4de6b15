// Production horizon march for sm_100a: one DEM pass of the hierarchical,
// adaptive ray march over a 128x128 tile x 1440 azimuths, one thread per ray
// (the drop-in for subpatch_hierarchy_kernel, cuda_backend.py:1007-1134; the
// per-ray core and its arithmetic contract are in march_core.cuh).
//
// Layout.  Working slopes are azimuth-major [A, P] so that a warp (32
// adjacent pixels of one tile row, one azimuth) reads and writes 128
// contiguous bytes; a transpose kernel produces the reference's pixel-major
// [P, A] at the end.  The first pass writes without reading (the reference
// resets the buffer to -inf before pass 0).
#include "march_core.cuh"

namespace ls200 {

struct MarchParams {
    const float *segments;  // [A, C, D, 18]
    int azimuth_count, center_count, dem_count;
    const float *primary_cells;
    int primary_width, primary_height;
    float primary_m6, primary_m9;
    const float *cells;   // sanitized level 0 + mips of the active DEM
    const float *bounds;  // four-cell bounds of those cells
    int width, height;
    int level_count;
    int4 levels[kMaxLevels];  // (cell offset, width, height, -)
    float m6, m7, m9, m10, radius;
    int tile_column, tile_row, tile_width, tile_height, subpatch, pass_index;
    float observer_elevation;
    float *slopes;  // [A, P]
    int first_pass;
    unsigned long long *counters;
};

// Level table shared by a block (every thread of a launch marches the same
// DEM at the same resolution).
struct SharedLevels {
    const LevelTable &t;
    __device__ __forceinline__ float side(int l) const { return t.side[l]; }
    __device__ __forceinline__ float fallback(int l) const { return t.fallback[l]; }
    __device__ __forceinline__ float out_step(int l) const { return t.out_step[l]; }
    __device__ __forceinline__ int4 cells(int l) const { return t.cells[l]; }
};

// Resident 128-thread blocks per SM the register budget is sized for.  With
// the f32x2 pairs and the Newton reciprocal, 9 (56 registers) marched 3.9 %
// faster than 10 (48 registers, whose spills had grown) and 3.6 % faster than
// 8 (64 registers) on site-scale tiles; 12 was slower.
#ifndef LS_MARCH_MIN_BLOCKS
#define LS_MARCH_MIN_BLOCKS 9
#endif
// Adjacent pixels of one azimuth in a warp (a power of two up to 32); the
// warp's other lanes take the next azimuths of the same pixels.  4 pixels x
// 8 azimuths marched 4.3 % faster than 32 pixels x 1 azimuth on site-scale
// tiles (8 px: 3.9 %, 16 px: 2.1 %), with the same results.
#ifndef LS_MARCH_LANES
#define LS_MARCH_LANES 4
#endif
constexpr int kMarchLanes = LS_MARCH_LANES;
static_assert(kMarchLanes >= 1 && kMarchLanes <= 32 && (kMarchLanes & (kMarchLanes - 1)) == 0,
              "LS_MARCH_LANES must be a power of two up to 32");

// Threads a pass launches for `pixels` x `azimuths` rays in this layout.
static long long march_threads(int pixels, int azimuths) {
    if (kMarchLanes == 32) return static_cast<long long>(pixels) * azimuths;
    const long long pixel_groups = (pixels + kMarchLanes - 1) / kMarchLanes;
    const long long azimuth_groups = (azimuths + 32 / kMarchLanes - 1) / (32 / kMarchLanes);
    return pixel_groups * azimuth_groups * 32;
}

template <bool kCount>
__global__ void __launch_bounds__(128, LS_MARCH_MIN_BLOCKS)
    march_pass_kernel(const __grid_constant__ MarchParams P) {
    __shared__ LevelTable table;
    const float column_res = hypot_fused(P.m6, P.m9);
    const float resolution = mean_resolution(P.m6, P.m7, P.m9, P.m10);
    if (threadIdx.x < P.level_count)
        fill_level(table, threadIdx.x, resolution, P.levels[threadIdx.x]);
    __syncthreads();

    const int pixel_count = P.tile_width * P.tile_height;
    const long long linear = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    int pixel, azimuth;
    if (kMarchLanes == 32) {
        if (linear >= static_cast<long long>(pixel_count) * P.azimuth_count) return;
        pixel = static_cast<int>(linear % pixel_count);
        azimuth = static_cast<int>(linear / pixel_count);
    } else {
        const long long warp = linear >> 5;
        const int lane = static_cast<int>(linear & 31);
        const long long pixel_groups = (pixel_count + kMarchLanes - 1) / kMarchLanes;
        const long long azimuth_group = warp / pixel_groups;
        const long long pixel_group = warp - azimuth_group * pixel_groups;
        pixel = static_cast<int>(pixel_group * kMarchLanes + lane % kMarchLanes);
        azimuth = static_cast<int>(azimuth_group * (32 / kMarchLanes) + lane / kMarchLanes);
        if (pixel >= pixel_count || azimuth >= P.azimuth_count) return;
    }
    const int row = pixel / P.tile_width;
    const int column = pixel % P.tile_width;
    float *out = P.slopes + static_cast<size_t>(azimuth) * pixel_count + pixel;
    // Pixels outside the primary DEM keep the initial -inf sentinel.
    if (P.tile_column + column >= P.primary_width || P.tile_row + row >= P.primary_height) {
        if (P.first_pass) *out = -INFINITY;
        return;
    }
    const float ratio = __fdiv_rn(hypot_fused(P.primary_m6, P.primary_m9), column_res);
    const RaySegment g = interpolate_segment(
        P.segments, P.center_count, P.dem_count, P.pass_index, azimuth, column, row,
        P.tile_column, P.tile_row, P.tile_width, P.subpatch, P.primary_width, P.primary_height,
        ratio);
    const float observer_z = __fadd_rn(
        bilinear(P.primary_cells, P.primary_width, P.primary_height,
                 static_cast<float>(P.tile_column + column),
                 static_cast<float>(P.tile_row + row)),
        P.observer_elevation);
    float current = -1e30f;
    if (!P.first_pass) {
        const float initial = *out;
        current = isinf(initial) ? -1e30f : initial;
    }
    const DemView dem{P.cells, P.bounds, P.width, P.height, P.level_count, resolution, column_res,
                      P.radius};
    unsigned visits = 0, samples = 0, steps = 0;
    current = march_dem<kCount, kReference>(SharedLevels{table}, dem, g, P.pass_index, observer_z,
                                       current, visits, samples, steps);
    *out = current > -1e29f ? current : -INFINITY;
    if (kCount) add_counters(P.counters, visits, samples, steps);
}

void march_pass_device(ls200_context *ctx, const MarchTile &tile, const ls200_dem *primary,
                       const ls200_dem *active, int pass_index, bool first_pass,
                       float *slopes_az_major) {
    // The clamped bilinear sample needs at least a 2x2 grid.
    LS_REQUIRE(primary->width >= 2 && primary->height >= 2 && active->width >= 2 &&
                   active->height >= 2,
               "DEMs must be at least 2x2 pixels");
    MarchParams P{};
    P.segments = tile.segments;
    P.azimuth_count = tile.azimuth_count;
    P.center_count = tile.center_count;
    P.dem_count = tile.dem_count;
    P.primary_cells = primary->cells;
    P.primary_width = primary->width;
    P.primary_height = primary->height;
    P.primary_m6 = primary->map_parameters[6];
    P.primary_m9 = primary->map_parameters[9];
    P.cells = active->cells;
    P.bounds = active->bounds;
    P.width = active->width;
    P.height = active->height;
    P.level_count = active->level_count;
    const int cells0 = active->width * active->height;
    for (int l = 0; l < active->level_count; ++l)
        P.levels[l] = make_int4(l == 0 ? 0 : cells0 + active->levels[l].offset,
                                active->levels[l].width, active->levels[l].height, 0);
    P.m6 = active->map_parameters[6];
    P.m7 = active->map_parameters[7];
    P.m9 = active->map_parameters[9];
    P.m10 = active->map_parameters[10];
    P.radius = static_cast<float>(active->projection[0]);
    P.tile_column = tile.tile_column;
    P.tile_row = tile.tile_row;
    P.tile_width = tile.tile_width;
    P.tile_height = tile.tile_height;
    P.subpatch = tile.subpatch;
    P.pass_index = pass_index;
    P.observer_elevation = tile.observer_elevation;
    P.slopes = slopes_az_major;
    P.first_pass = first_pass ? 1 : 0;
    P.counters = ctx->counters.as<unsigned long long>();
    const long long total =
        march_threads(tile.tile_width * tile.tile_height, tile.azimuth_count);
    const unsigned blocks = static_cast<unsigned>((total + 127) / 128);
    if (ctx->counting)
        march_pass_kernel<true><<<blocks, 128, 0, ctx->stream>>>(P);
    else
        march_pass_kernel<false><<<blocks, 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
}

}  // namespace ls200
