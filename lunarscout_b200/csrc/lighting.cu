// Lighting products against 1440-azimuth horizon tiles on sm_100a:
// sun fraction (float32 and byte), body-centre margin, PSR.
//
// Semantics follow src/lunarscout/_numba_horizon/lightmap_cpu.py:25-183 (the
// per-pixel FP64 east/north/up frame, float32 per time step, 16-slice solar
// disk of src/lunarscout/_numba_horizon/lightmap.py:15-29) and
// psr_cuda.py:57-186 (PSR).  Arithmetic is the reference CPU backend's, op by
// op (this file builds with --fmad=false); atan2f is CUDA's.
//
// Design: the per-pixel frame (FP64 trigonometry) is computed once per tile
// into 12 floats per pixel; the time loop is split into chunks so that a
// tile's 16384 pixels x T times fill all SMs; one thread owns one pixel of
// one chunk and writes time-major rows [t, 128*128] (coalesced across the
// warp).  Many tiles may share one launch (blockIdx.z).
#define LS200_LIGHTING_KERNELS
#include "internal.cuh"
#include "lighting.cuh"

namespace ls200 {

// Whether the disk constants are on a device yet.  Contexts on one device
// each hold only their own lock, so the flag has a lock of its own.
static std::mutex g_constants_lock;
static bool g_constants_ready[64] = {};

void ensure_lighting_constants(ls200_context *ctx) {
    std::lock_guard<std::mutex> hold(g_constants_lock);
    if (g_constants_ready[ctx->device]) return;
    // Half-chords of a 16-column disk of radius float32(0.27) deg
    // (lightmap.py:19-25), rounded once to float32; the normaliser is twice
    // their float32 running sum.
    float hc[16];
    float sum = 0.0f;
    for (int i = 0; i < 16; ++i) {
        const double x = 7.5 - i;
        hc[i] = static_cast<float>(std::sqrt(64.0 - x * x) / 8.0 * static_cast<double>(0.27f));
        sum = sum + hc[i];
    }
    const float max_photons = 2.0f * sum;
    LS_CUDA(cudaMemcpyToSymbol(c_half_circle, hc, sizeof hc));
    LS_CUDA(cudaMemcpyToSymbol(c_max_photons, &max_photons, sizeof max_photons));
    g_constants_ready[ctx->device] = true;
}

// FP64 east/north/up frame of one DEM pixel (lightmap_cpu.py:51-103).
__device__ Frame32 pixel_frame(const TileGeo &g, int column, int row, float height) {
    const double *gt = g.gt, *proj = g.proj;
    const double crs_x = gt[0] + gt[1] * column + gt[2] * row;
    const double crs_y = gt[3] + gt[4] * column + gt[5] * row;
    const double xp = crs_x - proj[4];
    const double yp = crs_y - proj[5];
    const double rho = sqrt(xp * xp + yp * yp);
    double latitude, longitude;
    if (rho <= 1e-12) {
        longitude = proj[2];
        latitude = proj[1];
    } else {
        const double c = 2.0 * atan2(rho, 2.0 * proj[3] * proj[0]);
        double sin_c, cos_c, sin_o, cos_o;
        sincos(c, &sin_c, &cos_c);
        sincos(proj[1], &sin_o, &cos_o);
        latitude = asin(cos_c * sin_o + yp * sin_c * cos_o / rho);
        longitude = proj[2] + atan2(xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c);
    }
    const double radius = proj[0] + static_cast<double>(height);
    double sin_lat, cos_lat, sin_lon, cos_lon;
    sincos(latitude, &sin_lat, &cos_lat);
    sincos(longitude, &sin_lon, &cos_lon);
    const double moon_x = radius * cos_lat * cos_lon;
    const double moon_y = radius * cos_lat * sin_lon;
    const double moon_z = radius * sin_lat;
    const double up_x = cos_lat * cos_lon, up_y = cos_lat * sin_lon, up_z = sin_lat;
    const double east_x = -sin_lon, east_y = cos_lon;
    const double north_x = -sin_lat * cos_lon, north_y = -sin_lat * sin_lon, north_z = cos_lat;
    Frame32 f;
    f.v[0] = static_cast<float>(east_x);   // r00
    f.v[1] = static_cast<float>(north_x);  // r01
    f.v[2] = static_cast<float>(up_x);     // r02
    f.v[3] = static_cast<float>(east_y);   // r10
    f.v[4] = static_cast<float>(north_y);  // r11
    f.v[5] = static_cast<float>(up_y);     // r12
    f.v[6] = 0.0f;                         // r20
    f.v[7] = static_cast<float>(north_z);  // r21
    f.v[8] = static_cast<float>(up_z);     // r22
    f.v[9] = static_cast<float>(-(moon_x * east_x + moon_y * east_y));
    f.v[10] = static_cast<float>(-(moon_x * north_x + moon_y * north_y + moon_z * north_z));
    f.v[11] = static_cast<float>(-(moon_x * up_x + moon_y * up_y + moon_z * up_z));
    return f;
}

__global__ void __launch_bounds__(128) frames_kernel(const __grid_constant__ LightingBatch B) {
    const int tile = blockIdx.y;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    const int sample = index % kPatch, line = index / kPatch;
    Frame32 f{};
    if (sample < g.valid_width && line < g.valid_height)
        f = pixel_frame(g, g.tile_x + sample, g.tile_y + line,
                        B.patch_dem[static_cast<size_t>(tile) * kPatch * kPatch + index]);
    float *dst = B.frames + (static_cast<size_t>(tile) * kPatch * kPatch + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) dst[k] = f.v[k];
}

// Per-thread window of staged horizon bins (stride 33 spreads the threads'
// windows over the 32 shared-memory banks).
constexpr int kWindowBins = 32;
constexpr int kWindowStride = kWindowBins + 1;

// Stage the bins that positions [k0, k1) of the launch's order read (kSpan
// bins from each step's first bin: 2 for the margin, 5 for the fraction)
// into `window`; returns the number staged (0: none) and sets `first`, the
// window's first bin.  In longitude order the body's azimuth moves
// monotonically across a chunk, so the bins between those of its first and
// last steps, plus the span and a margin of 2 on each side, cover it; a step
// outside them reads its row directly.
template <int kSpan>
__device__ __forceinline__ int stage_window(const LightingBatch &B, const Frame32 &f,
                                            const float *horizon, int k0, int k1, float *window,
                                            int &first) {
    if (!B.order || k1 <= k0) return 0;
    float azimuth_deg, elevation;
    const float *v = B.vectors + 3 * static_cast<size_t>(__ldg(B.order + k0));
    body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
    const int a = kSpan == 2 ? margin_position(azimuth_deg).left : sun_position(azimuth_deg).left;
    v = B.vectors + 3 * static_cast<size_t>(__ldg(B.order + k1 - 1));
    body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
    const int b = kSpan == 2 ? margin_position(azimuth_deg).left : sun_position(azimuth_deg).left;
    int arc = b - a;
    if (arc < 0) arc += kAzimuths;
    int start = arc <= kAzimuths / 2 ? a : b;
    if (arc > kAzimuths / 2) arc = kAzimuths - arc;
    start -= 2;
    if (start < 0) start += kAzimuths;
    if (arc + kSpan + 4 > kWindowBins) return 0;
    first = start;
    const int width = arc + kSpan + 4;
    for (int i = 0; i < width; ++i) {
        int bin = first + i;
        if (bin >= kAzimuths) bin -= kAzimuths;
        window[i] = __ldg(horizon + bin);
    }
    return width;
}

// Chunk length of an ordered launch: a chunk of c steps sweeps about
// c * 1440 / T bins; keep that to 20 so its bins fit the staged window.
static int ordered_chunk(int chunk, int time_count) {
    return std::min(chunk, std::max(16, (kWindowBins - 12) * time_count / kAzimuths));
}

template <int kSignal>
__global__ void __launch_bounds__(128) lighting_kernel(const __grid_constant__ LightingBatch B) {
    const int tile = blockIdx.z;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    const int sample = index % kPatch, line = index / kPatch;
    // Chunk blockIdx.y covers positions [k0, k1) of the launch's order.
    const int k0 = blockIdx.y * B.chunk;
    const int k1 = min(k0 + B.chunk, B.time_count);
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    const size_t tile_out = static_cast<size_t>(tile) * B.time_count * plane;
    if (sample >= g.valid_width || line >= g.valid_height) {
        for (int k = k0; k < k1; ++k) {
            const int t = B.order ? __ldg(B.order + k) : B.time_start + k;
            const size_t o = tile_out + static_cast<size_t>(t - B.time_start) * plane + index;
            if (kSignal == kSignalBytes) static_cast<uint8_t *>(B.out)[o] = 0;
            else static_cast<float *>(B.out)[o] = 0.0f;
        }
        return;
    }
    Frame32 f;
    const float *src = B.frames + (static_cast<size_t>(tile) * plane + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) f.v[k] = src[k];
    const float *horizon = B.horizons + (static_cast<size_t>(tile) * plane + index) * kAzimuths;
    __shared__ float windows[128 * kWindowStride];
    float *window = windows + threadIdx.x * kWindowStride;
    constexpr int kSpan = kSignal == kSignalMargin ? 2 : 5;
    int first = 0;
    const int width = stage_window<kSpan>(B, f, horizon, k0, k1, window, first);
    for (int k = k0; k < k1; ++k) {
        const int t = B.order ? __ldg(B.order + k) : B.time_start + k;
        const float *v = B.vectors + 3 * static_cast<size_t>(t);
        float azimuth_deg, elevation;
        body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
        const size_t o = tile_out + static_cast<size_t>(t - B.time_start) * plane + index;
        const BinPosition p = kSignal == kSignalMargin ? margin_position(azimuth_deg)
                                                       : sun_position(azimuth_deg);
        int offset = p.left - first;
        if (offset < 0) offset += kAzimuths;
        const bool staged = offset + kSpan <= width;
        if (kSignal == kSignalMargin) {
            static_cast<float *>(B.out)[o] =
                staged ? horizon_margin_bins(SharedBins{window, offset}, p.fraction, elevation)
                       : horizon_margin_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
        } else {
            const float visible =
                staged ? sun_fraction_bins(SharedBins{window, offset}, p.fraction, elevation)
                       : sun_fraction_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
            if (kSignal == kSignalBytes)
                static_cast<uint8_t *>(B.out)[o] =
                    static_cast<uint8_t>(static_cast<int>(__fmul_rn(255.0f, visible)));
            else
                static_cast<float *>(B.out)[o] = visible;
        }
    }
}

// PSR (psr_cuda.py:57-186): 255 unless a reduced vector's centre rises above
// the interpolated horizon minus 0.545/2 deg; exits at the first such vector.
__global__ void __launch_bounds__(128) psr_kernel(const __grid_constant__ LightingBatch B) {
    const int tile = blockIdx.z;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    const int sample = index % kPatch, line = index / kPatch;
    uint8_t *out = static_cast<uint8_t *>(B.out) + static_cast<size_t>(tile) * kPatch * kPatch;
    if (sample >= g.valid_width || line >= g.valid_height) {
        out[index] = 0;
        return;
    }
    Frame32 f;
    const float *src = B.frames + (static_cast<size_t>(tile) * kPatch * kPatch + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) f.v[k] = src[k];
    const float *horizon =
        B.horizons + (static_cast<size_t>(tile) * kPatch * kPatch + index) * kAzimuths;
    uint8_t is_psr = 255;
    for (int t = 0; t < B.time_count; ++t) {
        const float *v = B.vectors + 3 * static_cast<size_t>(t);
        float azimuth_deg, elevation;
        body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
        float position = __fmul_rn(azimuth_deg, 4.0f);
        if (position >= static_cast<float>(kAzimuths)) position = 0.0f;
        const int lower = static_cast<int>(position);
        const float fraction = __fsub_rn(position, static_cast<float>(lower));
        const int upper = lower + 1 >= kAzimuths ? 0 : lower + 1;
        const float h1 = __ldg(horizon + lower), h2 = __ldg(horizon + upper);
        const float h = __fadd_rn(h1, __fmul_rn(fraction, __fsub_rn(h2, h1)));
        if (__fsub_rn(elevation, h) > -0.2725f) {
            is_psr = 0;
            break;
        }
    }
    out[index] = is_psr;
}

// Diagnostic: sun fraction for given (azimuth, elevation) per horizon row
// (the reference's _sun_fraction_reference, lightmap.py:32-73).
__global__ void sun_fraction_kernel(const float *horizons, const float *azimuth_deg,
                                    const float *elevation_deg, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = sun_fraction(horizons + static_cast<size_t>(i) * kAzimuths, azimuth_deg[i],
                          elevation_deg[i]);
}

int lighting_chunk(ls200_context *ctx, int tiles, int time_count) {
    // Enough (pixel-block x chunk x tile) blocks for ~8 waves of 128-thread
    // blocks on every SM, chunks of at least 16 time steps.
    const int blocks_per_chunk = (kPatch * kPatch / 128) * tiles;
    const int want = ctx->props.multiProcessorCount * 16 * 8;
    int chunks = std::max(1, want / std::max(1, blocks_per_chunk));
    chunks = std::min(chunks, std::max(1, time_count / 16));
    return (time_count + chunks - 1) / chunks;
}

// window = the entries of `order` inside [t0, t0 + n), in order: one block,
// each thread counting and then copying a contiguous run of `order` at the
// offset given by a block scan of the counts.
constexpr int kOrderThreads = 1024;

__global__ void __launch_bounds__(kOrderThreads) order_window_kernel(
    const int *__restrict__ order, int count, int t0, int n, int *__restrict__ window) {
    __shared__ int sums[kOrderThreads];
    const int per = (count + kOrderThreads - 1) / kOrderThreads;
    const int begin = min(count, static_cast<int>(threadIdx.x) * per);
    const int end = min(count, begin + per);
    int mine = 0;
    for (int k = begin; k < end; ++k) {
        const int t = order[k];
        mine += (t >= t0 && t < t0 + n) ? 1 : 0;
    }
    sums[threadIdx.x] = mine;
    __syncthreads();
    for (int offset = 1; offset < kOrderThreads; offset <<= 1) {
        const int add = threadIdx.x >= static_cast<unsigned>(offset) ? sums[threadIdx.x - offset]
                                                                     : 0;
        __syncthreads();
        sums[threadIdx.x] += add;
        __syncthreads();
    }
    int position = sums[threadIdx.x] - mine;
    for (int k = begin; k < end; ++k) {
        const int t = order[k];
        if (t >= t0 && t < t0 + n) window[position++] = t;
    }
}

void lighting_launch(ls200_context *ctx, LightingBatch &B, int tiles, int signal,
                     const ls200_vectors *table) {
    ensure_lighting_constants(ctx);
    B.order = nullptr;
    if (table && table->order && signal != kSignalPsr) {
        if (B.time_start == 0 && B.time_count == table->count) {
            B.order = table->order;
        } else {
            order_window_kernel<<<1, kOrderThreads, 0, ctx->stream>>>(
                table->order, table->count, B.time_start, B.time_count, table->window);
            LS_CUDA(cudaGetLastError());
            B.order = table->window;
        }
    }
    dim3 grid_frames(kPatch * kPatch / 128, tiles);
    frames_kernel<<<grid_frames, 128, 0, ctx->stream>>>(B);
    LS_CUDA(cudaGetLastError());
    if (signal == kSignalPsr) {
        dim3 grid(kPatch * kPatch / 128, 1, tiles);
        psr_kernel<<<grid, 128, 0, ctx->stream>>>(B);
    } else {
        B.chunk = lighting_chunk(ctx, tiles, B.time_count);
        if (B.order) B.chunk = ordered_chunk(B.chunk, B.time_count);
        dim3 grid(kPatch * kPatch / 128, (B.time_count + B.chunk - 1) / B.chunk, tiles);
        if (signal == kSignalFraction)
            lighting_kernel<kSignalFraction><<<grid, 128, 0, ctx->stream>>>(B);
        else if (signal == kSignalBytes)
            lighting_kernel<kSignalBytes><<<grid, 128, 0, ctx->stream>>>(B);
        else
            lighting_kernel<kSignalMargin><<<grid, 128, 0, ctx->stream>>>(B);
    }
    LS_CUDA(cudaGetLastError());
}

__global__ void __launch_bounds__(128) directions_kernel(const __grid_constant__ LightingBatch B,
                                                         float2 *__restrict__ out) {
    const int tile = blockIdx.z;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    const int sample = index % kPatch, line = index / kPatch;
    const int t0 = B.time_start + blockIdx.y * B.chunk;
    const int t1 = min(t0 + B.chunk, B.time_start + B.time_count);
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    const size_t tile_out = static_cast<size_t>(tile) * B.time_count * plane;
    const bool valid = sample < g.valid_width && line < g.valid_height;
    Frame32 f;
    const float *src = B.frames + (static_cast<size_t>(tile) * plane + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) f.v[k] = src[k];
    for (int t = t0; t < t1; ++t) {
        float2 direction = make_float2(0.0f, 0.0f);
        if (valid) {
            const float *v = B.vectors + 3 * static_cast<size_t>(t);
            body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), direction.x, direction.y);
        }
        out[tile_out + static_cast<size_t>(t - B.time_start) * plane + index] = direction;
    }
}

void directions_launch(ls200_context *ctx, LightingBatch &B, int tiles, float2 *out) {
    LS_REQUIRE(tiles >= 1 && tiles <= kMaxBatchTiles, "1 to 32 tiles per launch");
    dim3 grid_frames(kPatch * kPatch / 128, tiles);
    frames_kernel<<<grid_frames, 128, 0, ctx->stream>>>(B);
    LS_CUDA(cudaGetLastError());
    B.chunk = lighting_chunk(ctx, tiles, B.time_count);
    dim3 grid(kPatch * kPatch / 128, (B.time_count + B.chunk - 1) / B.chunk, tiles);
    directions_kernel<<<grid, 128, 0, ctx->stream>>>(B, out);
    LS_CUDA(cudaGetLastError());
}

// Sun fraction at (azimuth, elevation) from a thread's staged window when it
// holds the five bins, else from the pixel's row.
__device__ __forceinline__ float staged_sun_fraction(const float *window, int first, int width,
                                                     const float *horizon, float azimuth_deg,
                                                     float elevation) {
    const BinPosition p = sun_position(azimuth_deg);
    int offset = p.left - first;
    if (offset < 0) offset += kAzimuths;
    return offset + 5 <= width
               ? sun_fraction_bins(SharedBins{window, offset}, p.fraction, elevation)
               : sun_fraction_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
}

// The same for the margin (two bins).
__device__ __forceinline__ float staged_margin(const float *window, int first, int width,
                                               const float *horizon, float azimuth_deg,
                                               float elevation) {
    const BinPosition p = margin_position(azimuth_deg);
    int offset = p.left - first;
    if (offset < 0) offset += kAzimuths;
    return offset + 2 <= width
               ? horizon_margin_bins(SharedBins{window, offset}, p.fraction, elevation)
               : horizon_margin_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
}

// Threshold bits of one signal of one body, word-major [tiles, words, 16384]
// (zeroed before the launch): bit t is set where signal >= threshold
// (kAtLeast) or signal < threshold.  kSpan 5 is the sun fraction, 2 the
// margin.  Each thread visits a chunk of the body's table in its longitude
// order with the chunk's bins staged, and sets the bits of its steps with
// atomicOr (other chunks own the word's other steps).  Each signal runs in
// its own body's order, so the Earth's reads are staged as well as the Sun's.
template <int kSpan, bool kAtLeast>
__global__ void __launch_bounds__(128) signal_bits_kernel(const __grid_constant__ LightingBatch B,
                                                          float threshold, int words,
                                                          uint32_t *__restrict__ bits) {
    const int tile = blockIdx.z;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    const int sample = index % kPatch, line = index / kPatch;
    if (sample >= g.valid_width || line >= g.valid_height) return;
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    uint32_t *tile_bits = bits + static_cast<size_t>(tile) * words * plane + index;
    const int k0 = blockIdx.y * B.chunk;
    const int k1 = min(k0 + B.chunk, B.time_count);
    Frame32 f;
    const float *src = B.frames + (static_cast<size_t>(tile) * plane + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) f.v[k] = src[k];
    const float *horizon = B.horizons + (static_cast<size_t>(tile) * plane + index) * kAzimuths;
    __shared__ float windows[128 * kWindowStride];
    float *window = windows + threadIdx.x * kWindowStride;
    int first = 0;
    const int width = stage_window<kSpan>(B, f, horizon, k0, k1, window, first);
    for (int k = k0; k < k1; ++k) {
        const int t = B.order ? __ldg(B.order + k) : k;
        const float *v = B.vectors + 3 * static_cast<size_t>(t);
        float azimuth_deg, elevation;
        body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
        const float value =
            kSpan == 5 ? staged_sun_fraction(window, first, width, horizon, azimuth_deg, elevation)
                       : staged_margin(window, first, width, horizon, azimuth_deg, elevation);
        const bool on = kAtLeast ? value >= threshold : value < threshold;
        if (on) atomicOr(tile_bits + static_cast<size_t>(t >> 5) * plane, 1u << (t & 31));
    }
}

// Zero `bits` ([tiles, words, 16384] words) and set the threshold bits of
// one signal: `table` (vectors and their longitude order, or NULL for time
// order) replaces the batch's vectors; the frames are already in place.
template <int kSpan, bool kAtLeast>
static void signal_bits_launch(ls200_context *ctx, LightingBatch B, int tiles,
                               const float *vectors, const int *order, float threshold,
                               int words, uint32_t *bits) {
    LS_CUDA(cudaMemsetAsync(bits, 0,
                            sizeof(uint32_t) * static_cast<size_t>(tiles) * words * kPatch * kPatch,
                            ctx->stream));
    B.vectors = vectors;
    B.order = order;
    B.chunk = lighting_chunk(ctx, tiles, B.time_count);
    if (B.order) B.chunk = ordered_chunk(B.chunk, B.time_count);
    dim3 grid(kPatch * kPatch / 128, (B.time_count + B.chunk - 1) / B.chunk, tiles);
    signal_bits_kernel<kSpan, kAtLeast><<<grid, 128, 0, ctx->stream>>>(B, threshold, words, bits);
    LS_CUDA(cudaGetLastError());
}

// Longest right-censored candidate run per start interval
// (nh/mission_duration.py:212-256), one thread per pixel over the bits.  For
// a run of true samples [rs, re] and a start window [ws, we) the candidate
// starts at max(rs, ws) when that lies in the window and accrues every
// sample's duration through re; the answer per interval is the maximum over
// runs.  Durations are summed in sample order in FP64 as the reference does
// (or read from exact prefix sums when every sample duration is an integer).
constexpr int kMaxDurationIntervals = 64;

struct DurationParams {
    const uint32_t *bits;        // [tiles, words, 16384] sun fraction >= threshold
    const uint32_t *earth_bits;  // the same for Earth margin >= threshold, or NULL
    const double *hours;   // [T] sample durations
    const double *prefix;  // [T + 1] exact prefix sums, or NULL
    const int2 *windows;   // [I] (first, end) sample indices of each start window
    float *out;            // [tiles, I, 16384]
    int words, time_count, interval_count, tiles, days;
    int2 valid[kMaxBatchTiles];
};

__device__ __forceinline__ double run_hours(const DurationParams &P, int first, int last) {
    if (P.prefix) return P.prefix[last + 1] - P.prefix[first];
    double sum = 0.0;
    for (int t = first; t <= last; ++t) sum += P.hours[t];
    return sum;
}

__global__ void __launch_bounds__(128) duration_kernel(const __grid_constant__ DurationParams P) {
    const int tile = blockIdx.y;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    double longest[kMaxDurationIntervals];
    for (int i = 0; i < P.interval_count; ++i) longest[i] = 0.0;
    const bool valid =
        index % kPatch < P.valid[tile].x && index / kPatch < P.valid[tile].y;
    if (valid) {
        // Word-major bits: word w of this pixel at row[w * plane].  The
        // condition is the Sun bit, and with Earth vectors also the Earth bit.
        const size_t offset = static_cast<size_t>(tile) * P.words * plane + index;
        const uint32_t *row = P.bits + offset;
        const uint32_t *earth_row = P.earth_bits ? P.earth_bits + offset : nullptr;
        int run_start = -1;
        for (int t = 0; t <= P.time_count; ++t) {
            const size_t word = static_cast<size_t>(t >> 5) * plane;
            const bool on = t < P.time_count && ((row[word] >> (t & 31)) & 1u) &&
                            (!earth_row || ((earth_row[word] >> (t & 31)) & 1u));
            if (on) {
                if (run_start < 0) run_start = t;
                continue;
            }
            if (run_start < 0) continue;
            const int run_end = t - 1;
            for (int i = 0; i < P.interval_count; ++i) {
                const int2 w = P.windows[i];
                const int first = max(run_start, w.x);
                if (first >= w.y || first > run_end) continue;
                const double d = run_hours(P, first, run_end);
                if (d > longest[i]) longest[i] = d;
            }
            run_start = -1;
        }
    }
    for (int i = 0; i < P.interval_count; ++i) {
        const double v = P.days ? longest[i] / 24.0 : longest[i];
        P.out[(static_cast<size_t>(tile) * P.interval_count + i) * plane + index] =
            static_cast<float>(v);
    }
}

void mission_duration_launch(ls200_context *ctx, LightingBatch &B, int tiles,
                             const float *earth, float sun_threshold, float earth_threshold,
                             uint32_t *bits, const double *hours, const double *prefix,
                             const int2 *windows, int interval_count, bool days, float *out,
                             const int *order, const int *earth_order) {
    LS_REQUIRE(tiles >= 1 && tiles <= kMaxBatchTiles, "1 to 32 tiles per launch");
    LS_REQUIRE(interval_count >= 1 && interval_count <= kMaxDurationIntervals,
               "1 to 64 start intervals");
    ensure_lighting_constants(ctx);
    dim3 grid_frames(kPatch * kPatch / 128, tiles);
    frames_kernel<<<grid_frames, 128, 0, ctx->stream>>>(B);
    LS_CUDA(cudaGetLastError());
    const int words = (B.time_count + 31) / 32;
    const size_t stream_words = static_cast<size_t>(tiles) * words * kPatch * kPatch;
    signal_bits_launch<5, true>(ctx, B, tiles, B.vectors, order, sun_threshold, words, bits);
    if (earth)
        signal_bits_launch<2, true>(ctx, B, tiles, earth, earth_order, earth_threshold, words,
                                    bits + stream_words);
    DurationParams P{};
    P.bits = bits;
    P.earth_bits = earth ? bits + stream_words : nullptr;
    P.hours = hours;
    P.prefix = prefix;
    P.windows = windows;
    P.out = out;
    P.words = words;
    P.time_count = B.time_count;
    P.interval_count = interval_count;
    P.tiles = tiles;
    P.days = days ? 1 : 0;
    for (int t = 0; t < tiles; ++t)
        P.valid[t] = make_int2(B.tiles[t].valid_width, B.tiles[t].valid_height);
    duration_kernel<<<dim3(kPatch * kPatch / 128, tiles), 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
}

// Per-pixel safe-haven reducer (safe_haven.py:75-243), one thread per pixel
// over the condition bits in time order.  The reference credits a low-Sun run
// to every month band in which one of its samples saw an Earth outage, with
// the run's length at each of its samples; run lengths only grow, so the
// credit equals the run's final (or right-censored) length, applied once
// when the run ends.  Per band the scratch holds the longest credited run and
// flags 1 (an outage sample), 2 (a sample without outage), 4 (the current run
// touched this band); the flags of the band in use are gathered in a
// register and stored when the band changes or a run ends.  Output: band
// hours = float32(longest) * float32(time_step_hours), NaN where the band saw
// no outage or nothing else (safe_haven.py:231-240) and outside the valid
// rectangle.
struct HavenParams {
    const uint32_t *low, *outage;  // [tiles, words, 16384]
    const int *month;              // [T] band of each time step, -1 for none
    int *longest;                  // [tiles, bands, 16384] scratch
    uint8_t *flags;                // [tiles, bands, 16384] scratch
    float *out;                    // [tiles, bands, 16384]
    float hours;
    int words, time_count, bands;
    int2 valid[kMaxBatchTiles];
};

__global__ void __launch_bounds__(128) haven_kernel(const __grid_constant__ HavenParams P) {
    const int tile = blockIdx.y;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    const size_t band0 = static_cast<size_t>(tile) * P.bands * plane + index;
    int *longest = P.longest + band0;
    uint8_t *flags = P.flags + band0;
    float *out = P.out + band0;
    const bool valid = index % kPatch < P.valid[tile].x && index / kPatch < P.valid[tile].y;
    if (!valid) {
        for (int b = 0; b < P.bands; ++b) out[b * plane] = __int_as_float(0x7fffffff);
        return;
    }
    for (int b = 0; b < P.bands; ++b) {
        longest[b * plane] = 0;
        flags[b * plane] = 0;
    }
    int run = 0;
    int lo = P.bands, hi = -1;       // bands the current run touched lie in [lo, hi]
    int cached = -1;                 // band whose flags sit in `bits`
    unsigned bits = 0u;
    auto store = [&]() {
        if (cached >= 0 && bits) flags[cached * plane] |= static_cast<uint8_t>(bits);
        bits = 0u;
    };
    auto credit = [&]() {
        store();
        for (int b = lo; b <= hi; ++b) {
            const unsigned f = flags[b * plane];
            if (f & 4u) {
                longest[b * plane] = max(longest[b * plane], run);
                flags[b * plane] = static_cast<uint8_t>(f & ~4u);
            }
        }
        lo = P.bands;
        hi = -1;
    };
    const size_t word0 = static_cast<size_t>(tile) * P.words * plane + index;
    for (int w = 0; w < P.words; ++w) {
        const uint32_t low_word = __ldg(P.low + word0 + w * plane);
        const uint32_t outage_word = __ldg(P.outage + word0 + w * plane);
        const int steps = min(32, P.time_count - w * 32);
        for (int j = 0; j < steps; ++j) {
            const bool low = (low_word >> j) & 1u;
            const bool outage = (outage_word >> j) & 1u;
            if (low) {
                ++run;
            } else {
                if (hi >= 0) credit();
                run = 0;
            }
            const int m = __ldg(P.month + w * 32 + j);
            if (m >= 0) {
                if (m != cached) {
                    store();
                    cached = m;
                }
                bits |= outage ? 1u : 2u;
                if (outage && low) {
                    bits |= 4u;
                    lo = min(lo, m);
                    hi = max(hi, m);
                }
            }
        }
    }
    if (hi >= 0) credit();  // the run still open at the end is right-censored
    store();
    for (int b = 0; b < P.bands; ++b) {
        const unsigned f = flags[b * plane];
        out[b * plane] = (f & 3u) == 3u
                             ? __fmul_rn(__int2float_rn(longest[b * plane]), P.hours)
                             : __int_as_float(0x7fffffff);
    }
}

void safe_haven_launch(ls200_context *ctx, LightingBatch &B, int tiles, const float *earth,
                       float sunlight_threshold, float earth_threshold, uint32_t *bits,
                       const int *month, int bands, float hours, int *longest,
                       uint8_t *flags, float *out, const int *order,
                       const int *earth_order) {
    LS_REQUIRE(tiles >= 1 && tiles <= kMaxBatchTiles, "1 to 32 tiles per launch");
    ensure_lighting_constants(ctx);
    dim3 grid_frames(kPatch * kPatch / 128, tiles);
    frames_kernel<<<grid_frames, 128, 0, ctx->stream>>>(B);
    LS_CUDA(cudaGetLastError());
    const int words = (B.time_count + 31) / 32;
    const size_t stream_words = static_cast<size_t>(tiles) * words * kPatch * kPatch;
    // Low Sun (fraction < threshold) in the Sun's order, Earth outage
    // (margin < threshold) in the Earth's (safe_haven.py:156-160).
    signal_bits_launch<5, false>(ctx, B, tiles, B.vectors, order, sunlight_threshold, words,
                                 bits);
    signal_bits_launch<2, false>(ctx, B, tiles, earth, earth_order, earth_threshold, words,
                                 bits + stream_words);
    HavenParams P{};
    P.low = bits;
    P.outage = bits + stream_words;
    P.month = month;
    P.longest = longest;
    P.flags = flags;
    P.out = out;
    P.hours = hours;
    P.words = words;
    P.time_count = B.time_count;
    P.bands = bands;
    for (int t = 0; t < tiles; ++t)
        P.valid[t] = make_int2(B.tiles[t].valid_width, B.tiles[t].valid_height);
    haven_kernel<<<dim3(kPatch * kPatch / 128, tiles), 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
}

// Earth-visibility fraction: per pixel, the share of time steps whose Earth
// margin (the a13 signal of lighting_kernel, lightmap_cpu.py:121-141) is >=
// threshold.  Each thread counts its pixel over one time chunk and adds the
// count to the pixel's counter; visibility_finalize divides by T (FP64, then
// rounded to float32).
__global__ void __launch_bounds__(128) visibility_kernel(const __grid_constant__ LightingBatch B,
                                                         float threshold,
                                                         unsigned *__restrict__ counts) {
    const int tile = blockIdx.z;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const TileGeo &g = B.tiles[tile];
    if (index % kPatch >= g.valid_width || index / kPatch >= g.valid_height) return;
    const size_t plane = static_cast<size_t>(kPatch) * kPatch;
    const int k0 = blockIdx.y * B.chunk;
    const int k1 = min(k0 + B.chunk, B.time_count);
    Frame32 f;
    const float *src = B.frames + (static_cast<size_t>(tile) * plane + index) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) f.v[k] = src[k];
    const float *horizon = B.horizons + (static_cast<size_t>(tile) * plane + index) * kAzimuths;
    // A count does not depend on the order of its steps: visit them in the
    // table's longitude order with the chunk's bins staged (as lighting_kernel).
    __shared__ float windows[128 * kWindowStride];
    float *window = windows + threadIdx.x * kWindowStride;
    int first = 0;
    const int width = stage_window<2>(B, f, horizon, k0, k1, window, first);
    unsigned count = 0;
    for (int k = k0; k < k1; ++k) {
        const int t = B.order ? __ldg(B.order + k) : k;
        const float *v = B.vectors + 3 * static_cast<size_t>(t);
        float azimuth_deg, elevation;
        body_direction(f, __ldg(v), __ldg(v + 1), __ldg(v + 2), azimuth_deg, elevation);
        const BinPosition p = margin_position(azimuth_deg);
        int offset = p.left - first;
        if (offset < 0) offset += kAzimuths;
        const float margin =
            offset + 2 <= width
                ? horizon_margin_bins(SharedBins{window, offset}, p.fraction, elevation)
                : horizon_margin_bins(GlobalBins{horizon, p.left}, p.fraction, elevation);
        count += margin >= threshold ? 1u : 0u;
    }
    if (count) atomicAdd(counts + static_cast<size_t>(tile) * plane + index, count);
}

__global__ void visibility_finalize(const unsigned *__restrict__ counts, int n, int time_count,
                                    const int2 *__restrict__ valid, float *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int tile = i / (kPatch * kPatch), index = i % (kPatch * kPatch);
    const bool inside = index % kPatch < valid[tile].x && index / kPatch < valid[tile].y;
    out[i] = inside ? static_cast<float>(static_cast<double>(counts[i]) / time_count)
                    : __int_as_float(0x7fffffff);
}

void visibility_launch(ls200_context *ctx, LightingBatch &B, int tiles, float threshold,
                       unsigned *counts, int2 *valid, float *out, const int *order) {
    LS_REQUIRE(tiles >= 1 && tiles <= kMaxBatchTiles, "1 to 32 tiles per launch");
    ensure_lighting_constants(ctx);
    B.order = order;
    const int n = tiles * kPatch * kPatch;
    LS_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned) * n, ctx->stream));
    dim3 grid_frames(kPatch * kPatch / 128, tiles);
    frames_kernel<<<grid_frames, 128, 0, ctx->stream>>>(B);
    LS_CUDA(cudaGetLastError());
    B.chunk = lighting_chunk(ctx, tiles, B.time_count);
    if (B.order) B.chunk = ordered_chunk(B.chunk, B.time_count);
    dim3 grid(kPatch * kPatch / 128, (B.time_count + B.chunk - 1) / B.chunk, tiles);
    visibility_kernel<<<grid, 128, 0, ctx->stream>>>(B, threshold, counts);
    LS_CUDA(cudaGetLastError());
    visibility_finalize<<<(n + 255) / 256, 256, 0, ctx->stream>>>(counts, n, B.time_count, valid,
                                                                  out);
    LS_CUDA(cudaGetLastError());
}

void sun_fraction_launch(ls200_context *ctx, const float *horizons, const float *azimuth_deg,
                         const float *elevation_deg, int n, float *out) {
    ensure_lighting_constants(ctx);
    sun_fraction_kernel<<<(n + 127) / 128, 128, 0, ctx->stream>>>(horizons, azimuth_deg,
                                                                  elevation_deg, n, out);
    LS_CUDA(cudaGetLastError());
}

}  // namespace ls200
