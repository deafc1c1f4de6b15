// Lighting kernels' shared types and per-sample device arithmetic (included
// by lighting.cu and lighting_api.cu).  Arithmetic follows the reference CPU
// backend (src/lunarscout/_numba_horizon/lightmap_cpu.py:105-183) operation by
// operation; the translation units build with --fmad=false.
#pragma once

#include "internal.cuh"

// A Moon-ME vector table resident on the device (ls200_vectors_create).
struct ls200_vectors {
    ls200_context *ctx = nullptr;
    float *data = nullptr;  // device [count, 3]
    int count = 0;
    // device [count]: time indices sorted by the vector's longitude
    // atan2(y, x).  For a polar site the body's local azimuth follows its
    // longitude, so in this order consecutive steps read neighbouring
    // horizon bins.
    int *order = nullptr;
    int *window = nullptr;  // device [count]: one launch's sub-range of `order`
};

namespace ls200 {

constexpr int kPatch = 128;
constexpr int kAzimuths = 1440;
constexpr int kMaxBatchTiles = 32;
enum { kSignalFraction = 0, kSignalBytes = 1, kSignalMargin = 2, kSignalPsr = 3 };

struct Frame32 {
    float v[12];  // r00 r01 r02 r10 r11 r12 r20 r21 r22 tx ty tz
};

struct TileGeo {
    double gt[6];
    double proj[6];
    int tile_x, tile_y, valid_width, valid_height;
};

struct LightingBatch {
    TileGeo tiles[kMaxBatchTiles];
    const float *patch_dem;  // [tiles, 128, 128] (zero outside the valid rect)
    const float *horizons;   // [tiles, 128, 128, 1440] degrees
    const float *vectors;    // [T, 3] float32 Moon-ME metres
    float *frames;           // [tiles, 16384, 12]
    void *out;               // [tiles, time_count, 16384] (PSR: [tiles, 16384])
    int time_start, time_count, chunk;
    // [time_count] the launch's time indices in processing order, or NULL
    // for time order; outputs stay in time order either way.
    const int *order;
};

// With `table` (the vector table of the launch), fraction / byte / margin
// launches visit their time steps in the table's longitude order.
void lighting_launch(ls200_context *ctx, LightingBatch &batch, int tiles, int signal,
                     const ls200_vectors *table = nullptr);
void sun_fraction_launch(ls200_context *ctx, const float *horizons, const float *azimuth_deg,
                         const float *elevation_deg, int n, float *out);
void ensure_lighting_constants(ls200_context *ctx);
// Per-pixel frames of the batch's tiles, then the Sun's (azimuth deg,
// elevation deg) at every pixel and time step of [time_start, +time_count):
// out [tiles, time_count, 16384] (zero outside the valid rectangle).
void directions_launch(ls200_context *ctx, LightingBatch &batch, int tiles, float2 *out);
// The mission-duration product fused with the lighting: per-pixel condition
// bits (sun fraction >= sun_threshold [and, with `earth`, Earth margin >=
// earth_threshold]) into `bits` ([tiles, ceil(T/32), 16384] words per
// signal: room for two with `earth`), then the longest right-censored run
// per start interval into out [tiles, I, 16384] (hours, or days).  hours:
// device [T] sample durations; prefix: device [T + 1] exact prefix sums or
// NULL; windows: device [I] (first, end) sample indices of each start
// window; order / earth_order: the Sun's / Earth's table in longitude order
// (NULL: time order), the order in which each signal is evaluated.
void mission_duration_launch(ls200_context *ctx, LightingBatch &batch, int tiles,
                             const float *earth, float sun_threshold, float earth_threshold,
                             uint32_t *bits, const double *hours, const double *prefix,
                             const int2 *windows, int interval_count, bool days, float *out,
                             const int *order, const int *earth_order);

// The safe-haven product fused with the lighting: low-Sun and Earth-outage
// bits ([2, tiles, ceil(T/32), 16384] words in `bits`), then per pixel and
// month band the longest low-Sun run that overlapped an outage in that band,
// in hours, into out [tiles, bands, 16384] (NaN where the band is ill-posed).
// month: device [T] band index per time step (-1 for none); longest and
// flags: device scratch [tiles, bands, 16384]; order / earth_order: the
// Sun's / Earth's table in longitude order (NULL: time order), the order in
// which each body's bits are evaluated.
void safe_haven_launch(ls200_context *ctx, LightingBatch &batch, int tiles, const float *earth,
                       float sunlight_threshold, float earth_threshold, uint32_t *bits,
                       const int *month, int bands, float hours, int *longest,
                       uint8_t *flags, float *out, const int *order, const int *earth_order);

// Earth-visibility fraction: per pixel the share of the batch's time steps
// whose Earth margin is >= threshold (degrees), into out [tiles, 16384] (NaN
// outside the valid rectangle).  counts: device scratch [tiles, 16384];
// valid: device [tiles] (valid width, valid height); order: the table's
// longitude order of the time steps (NULL: time order).
void visibility_launch(ls200_context *ctx, LightingBatch &batch, int tiles, float threshold,
                       unsigned *counts, int2 *valid, float *out, const int *order);

#ifdef LS200_LIGHTING_KERNELS
// Slice half-heights and their normaliser (set by ensure_lighting_constants).
__constant__ float c_half_circle[16];
__constant__ float c_max_photons;

constexpr float kRadToDeg = 57.29577951308232f;  // float32(180/pi)
constexpr float kTwoPi = 6.283185307179586f;      // float32(2 pi)

// Azimuth (deg, [0, 360)) and elevation (deg) of a float32 Moon-ME vector in
// a pixel's frame (lightmap_cpu.py:105-120).
// The east and north components are computed as one f32x2 pair (sm_100),
// each lane rounding as the scalar __fmul_rn / __fadd_rn does.
__device__ __forceinline__ void body_direction(const Frame32 &f, float vx, float vy, float vz,
                                               float &azimuth_deg, float &elevation) {
    const float2 xy = __fadd2_rn(
        __fadd2_rn(__fadd2_rn(__fmul2_rn(make_float2(vx, vx), make_float2(f.v[0], f.v[1])),
                              __fmul2_rn(make_float2(vy, vy), make_float2(f.v[3], f.v[4]))),
                   __fmul2_rn(make_float2(vz, vz), make_float2(f.v[6], f.v[7]))),
        make_float2(f.v[9], f.v[10]));
    const float ex = xy.x, ey = xy.y;
    const float ez = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, f.v[2]), __fmul_rn(vy, f.v[5])),
                                         __fmul_rn(vz, f.v[8])), f.v[11]);
    const float2 squares = __fmul2_rn(xy, xy);
    const float horizontal = __fsqrt_rn(__fadd_rn(squares.x, squares.y));
    elevation = __fmul_rn(atan2f(ez, horizontal), kRadToDeg);
    float azimuth = atan2f(ex, ey);
    if (azimuth < 0.0f) azimuth = __fadd_rn(azimuth, kTwoPi);
    azimuth_deg = __fmul_rn(azimuth, kRadToDeg);
}

// The signals read the horizon bins left, left+1, ... (wrapped at 1440)
// through a bin accessor: GlobalBins reads the pixel's row, SharedBins a
// window of it staged in shared memory.  Both return the same values.
struct GlobalBins {
    const float *horizon;
    int left;
    __device__ __forceinline__ float operator()(int k) const {
        int b = left + k;
        if (b >= kAzimuths) b -= kAzimuths;
        return __ldg(horizon + b);
    }
};
struct SharedBins {
    const float *window;
    int offset;  // position of bin `left` in the window
    __device__ __forceinline__ float operator()(int k) const { return window[offset + k]; }
};

// First bin and interpolation fraction of the margin (2 bins).
struct BinPosition {
    int left;
    float fraction;
};
__device__ __forceinline__ BinPosition margin_position(float azimuth_deg) {
    const float position = __fmul_rn(azimuth_deg, 4.0f);
    int left = static_cast<int>(position);
    const float fraction = __fsub_rn(position, static_cast<float>(left));
    if (left >= kAzimuths) left -= kAzimuths;
    return BinPosition{left, fraction};
}

// Body-centre elevation minus the horizon interpolated at its azimuth
// (lightmap_cpu.py:121-141).
template <class Bins>
__device__ __forceinline__ float horizon_margin_bins(const Bins &bin, float fraction,
                                                     float elevation) {
    const float hl = bin(0), hr = bin(1);
    return __fsub_rn(elevation, __fadd_rn(hl, __fmul_rn(fraction, __fsub_rn(hr, hl))));
}

__device__ __forceinline__ float horizon_margin(const float *horizon, float azimuth_deg,
                                                float elevation) {
    const BinPosition p = margin_position(azimuth_deg);
    return horizon_margin_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
}

// Visible fraction of the solar disk: 16 vertical slices of a 0.27-deg disk
// against the linearly interpolated horizon, float32 accumulation
// (lightmap.py:32-73, lightmap_cpu.py:142-183).
//
// Exact shortcut: the 16 slices read bins left .. left+4 and interpolate (or,
// for the first slices, extrapolate by less than one bin) between them, so
// every slice's horizon lies within [min - span, max + span] of those bins.
// When that interval is clear of the whole disk by 1e-3 deg (far above the
// float32 rounding of degrees), every slice is fully lit (the float32 sum of
// the 2c_k is then exactly the normaliser: fraction 1) or fully dark
// (fraction 0), and the loop is skipped.
// First bin and fraction of the disk's first slice (the slices then read
// bins left .. left+4: 16 steps of 0.135 bin from a fraction below 1).
__device__ __forceinline__ BinPosition sun_position(float azimuth_deg) {
    const float left_position = __fmul_rn(__fsub_rn(__fsub_rn(azimuth_deg, 0.27f), 0.125f), 4.0f);
    int left = static_cast<int>(left_position);
    const float fraction = __fsub_rn(left_position, static_cast<float>(left));
    if (left < 0) left += kAzimuths;
    else if (left >= kAzimuths) left -= kAzimuths;
    return BinPosition{left, fraction};
}

template <class Bins>
__device__ __forceinline__ float sun_fraction_bins(const Bins &bin, float fraction,
                                                   float elevation) {
    {
        float lo = bin(0), hi = lo;
#pragma unroll
        for (int k = 1; k <= 4; ++k) {
            const float h = bin(k);
            lo = fminf(lo, h);
            hi = fmaxf(hi, h);
        }
        const float span = hi - lo;
        const float cmax = c_half_circle[7];
        if (hi + span <= elevation - cmax - 1e-3f) return 1.0f;
        if (lo - span >= elevation + cmax + 1e-3f) return 0.0f;
    }
    int right = 1;
    float left_elevation = bin(0);
    float right_elevation = bin(1);
    float delta = __fsub_rn(right_elevation, left_elevation);
    float photons = 0.0f;
#pragma unroll
    for (int slice = 0; slice < 16; ++slice) {
        const float h = __fadd_rn(__fmul_rn(fraction, delta), left_elevation);
        const float column = c_half_circle[slice];
        const float sun_top = __fadd_rn(elevation, column);
        if (h < sun_top) {
            float angle = __fsub_rn(sun_top, h);
            const float height = __fadd_rn(column, column);
            if (angle > height) angle = height;
            photons = __fadd_rn(photons, angle);
        }
        fraction = __fadd_rn(fraction, 0.135f);
        if (fraction >= 1.0f) {
            ++right;
            left_elevation = right_elevation;
            right_elevation = bin(right);
            delta = __fsub_rn(right_elevation, left_elevation);
            fraction = __fsub_rn(fraction, 1.0f);
        }
    }
    return __fdiv_rn(photons, c_max_photons);
}

__device__ __forceinline__ float sun_fraction(const float *horizon, float azimuth_deg,
                                              float elevation) {
    const BinPosition p = sun_position(azimuth_deg);
    return sun_fraction_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
}
#endif

}  // namespace ls200
