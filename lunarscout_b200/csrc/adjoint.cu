// The DEM adjoint of a time-integrated sun fraction (no reference
// counterpart; the differentiable model is this project's).
//
// Loss = sum over tiles and pixels of w * mean over time of F(u),
//   u = (el - h) / r,   F(u) = (acos(-u) + u sqrt(1 - u^2)) / pi  (|u| <= 1),
// the visible fraction of a sun disk of radius r above a locally level
// horizon line, h the horizon (degrees) interpolated at the sun's azimuth
// exactly as the reference's margin signal does (nh/lightmap_cuda.py:125-145:
// bin = az * 4, linear between bin and bin + 1, wrapping at 1440), with h
// clamped below at -90 deg.  The reference's own fraction (16 vertical slices
// against the interpolated horizon) is piecewise constant in h; F is its
// smooth counterpart, so the gradient exists.
//
// Forward: the persistent batched march of the tiles with per-ray argmax
// checkpoints (the winning level-0 sample's position, distance, slope, pass
// and near flag: 17 bytes per ray, not the ray), the sun direction per pixel
// and time (the lighting frames), then the loss in FP64.
// Backward: dL/dh per (pixel, azimuth) from the time sum, then per ray
// dL/dslope = dL/dh * (180/pi) / (1 + slope^2) and, through the winning
// sample, into the four bilinear corners of its height and the observer's
// own terrain height (FP64 atomics).  The sun direction's dependence on the
// local height (below 1e-9 deg per metre at 1 AU) is left out.
#include "lighting.cuh"

#include <cmath>
#include <vector>

namespace ls200 {

struct AdjointState {
    DeviceBuffer horizons;      // [tiles, 16384, A] degrees
    DeviceBuffer checkpoints;   // [tiles, 16384, A] float4
    DeviceBuffer flags;         // [tiles, 16384, A] uint8
    DeviceBuffer directions;    // [tiles, T, 16384] float2 (azimuth, elevation) deg
    DeviceBuffer patches;       // [tiles, 128, 128] heights for the lighting frames
    DeviceBuffer weights;       // [tiles, 16384]
    DeviceBuffer gradient;      // [tiles, 16384, A] double: dL/dh
    DeviceBuffer replayed;      // [tiles, 16384, A] double horizons of the last replay
    DeviceBuffer loss;          // 1 double
    bool use_replayed = false;  // the backward differentiates the last replay
    std::vector<ls200_dem *> dems;  // the shared DEM stack, primary first
    std::vector<int2> origins;      // tile origins (column, row)
    std::vector<float> observer;    // observer elevation per tile
    int tile_count = 0, azimuth_count = 0, time_count = 0;
    double radius_deg = 0.0;
    bool ready = false;
};

void release_adjoint_state(ls200_context *ctx) {
    delete ctx->adjoint;
    ctx->adjoint = nullptr;
}

static AdjointState &adjoint_of(ls200_context *ctx) {
    if (!ctx->adjoint) ctx->adjoint = new AdjointState();
    return *ctx->adjoint;
}

__global__ void gather_patches_kernel(const float *__restrict__ level0, int width, int height,
                                      const int2 *__restrict__ origins, float *__restrict__ out) {
    const int tile = blockIdx.y;
    const int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= kPatch * kPatch) return;
    const int2 o = origins[tile];
    const int x = o.x + index % kPatch, y = o.y + index / kPatch;
    out[static_cast<size_t>(tile) * kPatch * kPatch + index] =
        x < width && y < height ? level0[static_cast<size_t>(y) * width + x] : 0.0f;
}

// Horizon (deg) at the sun azimuth: left bin, fraction and the two values,
// each clamped below at -90.
struct HorizonAt {
    int left, right;
    double fraction, value;
    bool left_live, right_live;
};

template <class T>
__device__ __forceinline__ HorizonAt horizon_at(const T *__restrict__ row, int azimuth_count,
                                                float azimuth_deg) {
    HorizonAt h;
    const double position = static_cast<double>(azimuth_deg) * (azimuth_count / 360.0);
    h.left = static_cast<int>(position);
    h.fraction = position - h.left;
    if (h.left >= azimuth_count) h.left -= azimuth_count;
    h.right = h.left + 1 >= azimuth_count ? 0 : h.left + 1;
    const double hl = static_cast<double>(row[h.left]);
    const double hr = static_cast<double>(row[h.right]);
    h.left_live = hl > -90.0;
    h.right_live = hr > -90.0;
    const double l = h.left_live ? hl : -90.0, r = h.right_live ? hr : -90.0;
    h.value = l + h.fraction * (r - l);
    return h;
}

__device__ __forceinline__ double disk_fraction(double u) {
    if (u >= 1.0) return 1.0;
    if (u <= -1.0) return 0.0;
    return (acos(-u) + u * sqrt(1.0 - u * u)) / M_PI;
}

__device__ __forceinline__ double disk_fraction_slope(double u) {
    return fabs(u) >= 1.0 ? 0.0 : (2.0 / M_PI) * sqrt(1.0 - u * u);
}

struct LossParams {
    const float *horizons;
    const double *replayed;  // used instead of `horizons` when not NULL
    const float2 *directions;
    const float *weights;
    double *gradient;  // backward only
    double *loss;      // forward only
    int2 valid[kMaxBatchTiles];  // valid width, height per tile
    int azimuth_count, time_count;
    double radius_deg, scale;  // scale = grad_output / time_count
};

__global__ void __launch_bounds__(128) loss_kernel(const __grid_constant__ LossParams P) {
    const int tile = blockIdx.y;
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    double value = 0.0;
    if (pixel < kPatch * kPatch && pixel % kPatch < P.valid[tile].x &&
        pixel / kPatch < P.valid[tile].y) {
        const float w = P.weights[static_cast<size_t>(tile) * kPatch * kPatch + pixel];
        if (w != 0.0f) {
            const size_t base =
                (static_cast<size_t>(tile) * kPatch * kPatch + pixel) * P.azimuth_count;
            const float2 *dir = P.directions + static_cast<size_t>(tile) * P.time_count * kPatch *
                                                   kPatch + pixel;
            double sum = 0.0;
            for (int t = 0; t < P.time_count; ++t) {
                const float2 d = dir[static_cast<size_t>(t) * kPatch * kPatch];
                const HorizonAt h = P.replayed ? horizon_at(P.replayed + base, P.azimuth_count, d.x)
                                               : horizon_at(P.horizons + base, P.azimuth_count, d.x);
                sum += disk_fraction((static_cast<double>(d.y) - h.value) / P.radius_deg);
            }
            value = static_cast<double>(w) * sum / P.time_count;
        }
    }
    // Block sum, then one atomic per block.
    __shared__ double partial[4];
    for (int offset = 16; offset > 0; offset >>= 1)
        value += __shfl_down_sync(0xffffffffu, value, offset);
    if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = value;
    __syncthreads();
    // One partial per block, summed in a fixed order by sum_partials_kernel,
    // so that the loss is the same bits on every call.
    if (threadIdx.x == 0)
        P.loss[1 + blockIdx.y * gridDim.x + blockIdx.x] =
            partial[0] + partial[1] + partial[2] + partial[3];
}

__global__ void sum_partials_kernel(double *loss, int count) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double total = 0.0;
    for (int i = 0; i < count; ++i) total += loss[1 + i];
    loss[0] = total;
}

// loss_kernel + the ordered sum into loss[0] (loss holds 1 + blocks doubles).
static void launch_loss(ls200_context *ctx, const LossParams &P, int tile_count) {
    const int blocks_per_tile = kPatch * kPatch / 128;
    loss_kernel<<<dim3(blocks_per_tile, tile_count), 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
    sum_partials_kernel<<<1, 32, 0, ctx->stream>>>(P.loss, blocks_per_tile * tile_count);
    LS_CUDA(cudaGetLastError());
}

// dL/dh[pixel, azimuth] (each thread owns one pixel's row; zeroes it first).
__global__ void __launch_bounds__(128) horizon_gradient_kernel(const __grid_constant__ LossParams P) {
    const int tile = blockIdx.y;
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= kPatch * kPatch) return;
    const size_t base = (static_cast<size_t>(tile) * kPatch * kPatch + pixel) * P.azimuth_count;
    double *grad = P.gradient + base;
    for (int a = 0; a < P.azimuth_count; ++a) grad[a] = 0.0;
    if (pixel % kPatch >= P.valid[tile].x || pixel / kPatch >= P.valid[tile].y) return;
    const float w = P.weights[static_cast<size_t>(tile) * kPatch * kPatch + pixel];
    if (w == 0.0f) return;
    const float2 *dir =
        P.directions + static_cast<size_t>(tile) * P.time_count * kPatch * kPatch + pixel;
    const double factor = static_cast<double>(w) * P.scale / P.radius_deg;
    for (int t = 0; t < P.time_count; ++t) {
        const float2 d = dir[static_cast<size_t>(t) * kPatch * kPatch];
        const HorizonAt h = P.replayed ? horizon_at(P.replayed + base, P.azimuth_count, d.x)
                                       : horizon_at(P.horizons + base, P.azimuth_count, d.x);
        const double u = (static_cast<double>(d.y) - h.value) / P.radius_deg;
        const double g = -factor * disk_fraction_slope(u);  // dL/dh at the interpolated h
        if (g == 0.0) continue;
        if (h.left_live) grad[h.left] += g * (1.0 - h.fraction);
        if (h.right_live) grad[h.right] += g * h.fraction;
    }
}

// Bilinear sample weights of the reference's clamped bilinear (in double,
// from the float32 clamp the march applies).
struct Corners {
    int index[4];
    double weight[4];
};

__device__ __forceinline__ Corners bilinear_corners(int width, int height, float column, float row) {
    const float cmax = __fsub_rn(static_cast<float>(width), 1.0001f);
    const float rmax = __fsub_rn(static_cast<float>(height), 1.0001f);
    column = column > 0.0f ? column : 0.0f;
    column = column < cmax ? column : cmax;
    row = row > 0.0f ? row : 0.0f;
    row = row < rmax ? row : rmax;
    const int x0 = static_cast<int>(floorf(column)), y0 = static_cast<int>(floorf(row));
    const int x1 = min(x0 + 1, width - 1), y1 = min(y0 + 1, height - 1);
    const double tx = static_cast<double>(column) - x0, ty = static_cast<double>(row) - y0;
    Corners c;
    c.index[0] = y0 * width + x0;
    c.index[1] = y0 * width + x1;
    c.index[2] = y1 * width + x0;
    c.index[3] = y1 * width + x1;
    c.weight[0] = (1.0 - tx) * (1.0 - ty);
    c.weight[1] = tx * (1.0 - ty);
    c.weight[2] = (1.0 - tx) * ty;
    c.weight[3] = tx * ty;
    return c;
}

struct ScatterDem {
    const float *level0;
    double *grad;
    int width, height;
    double radius;
};

struct ScatterParams {
    const float4 *checkpoints;
    const uint8_t *flags;
    const double *gradient;
    ScatterDem dems[8];
    int2 origins[kMaxBatchTiles];
    float observer[kMaxBatchTiles];
    int azimuth_count;
    long long rays_per_tile, total_rays;
};

// The winning sample of one ray, re-evaluated in FP64 at the DEMs' current
// heights: its slope and the slope's partials with respect to the sample's
// terrain height and the observer's (the reference's near-field and
// spherical slope formulas, nh/cuda_backend.py:812-830), with the bilinear
// corners of both heights.
struct SampleTerms {
    double slope, d_height, d_observer;
    Corners height_corners, observer_corners;
    int pass;
};

__device__ __forceinline__ SampleTerms sample_terms(const ScatterParams &P, long long ray,
                                                    uint8_t flag) {
    SampleTerms s;
    const int tile = static_cast<int>(ray / P.rays_per_tile);
    const int pixel = static_cast<int>((ray - tile * P.rays_per_tile) / P.azimuth_count);
    const float4 c = P.checkpoints[ray];
    s.pass = flag >> 1;
    const bool near = flag & 1;
    const ScatterDem &dem = P.dems[s.pass];
    const ScatterDem &primary = P.dems[0];
    s.height_corners = bilinear_corners(dem.width, dem.height, c.x, c.y);
    double height = 0.0;
    for (int k = 0; k < 4; ++k)
        height += s.height_corners.weight[k] * dem.level0[s.height_corners.index[k]];
    const int column = P.origins[tile].x + pixel % kPatch;
    const int row = P.origins[tile].y + pixel / kPatch;
    s.observer_corners = bilinear_corners(primary.width, primary.height,
                                          static_cast<float>(column), static_cast<float>(row));
    double observer_z = P.observer[tile];
    for (int k = 0; k < 4; ++k)
        observer_z += s.observer_corners.weight[k] * primary.level0[s.observer_corners.index[k]];
    const double distance = c.z;
    if (near) {
        s.slope = (height - observer_z) / distance;
        s.d_height = 1.0 / distance;
        s.d_observer = -1.0 / distance;
    } else {
        const double radius = dem.radius;
        const double rho = radius + observer_z;
        const double point = radius + height;
        const double z = (point * point - rho * rho - distance * distance) / (2.0 * rho);
        const double lx2 = distance * distance - z * z;
        const double x = lx2 > 0.0 ? sqrt(lx2) : 1e-6;
        const double dslope_dz = lx2 > 0.0 ? distance * distance / (lx2 * x) : 1e6;
        s.slope = z / x;
        s.d_height = dslope_dz * point / rho;
        s.d_observer = dslope_dz * (-1.0 - z / rho);
    }
    return s;
}

__global__ void __launch_bounds__(128) scatter_kernel(const __grid_constant__ ScatterParams P) {
    const long long ray = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ray >= P.total_rays) return;
    const double g = P.gradient[ray];
    const uint8_t flag = P.flags[ray];
    if (g == 0.0 || flag == 0xff) return;
    const SampleTerms s = sample_terms(P, ray, flag);
    const double g_slope = g * (180.0 / M_PI) / (1.0 + s.slope * s.slope);
    const ScatterDem &dem = P.dems[s.pass];
    const ScatterDem &primary = P.dems[0];
    for (int k = 0; k < 4; ++k) {
        if (s.height_corners.weight[k] != 0.0)
            atomicAdd(dem.grad + s.height_corners.index[k],
                      g_slope * s.d_height * s.height_corners.weight[k]);
        if (s.observer_corners.weight[k] != 0.0)
            atomicAdd(primary.grad + s.observer_corners.index[k],
                      g_slope * s.d_observer * s.observer_corners.weight[k]);
    }
}

// Horizons (degrees, FP64) of every ray from its recorded winning sample at
// the DEMs' current heights: the march's discrete choices held fixed.
__global__ void __launch_bounds__(128) replay_kernel(const __grid_constant__ ScatterParams P,
                                                    double *__restrict__ horizons) {
    const long long ray = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ray >= P.total_rays) return;
    const uint8_t flag = P.flags[ray];
    if (flag == 0xff) {
        horizons[ray] = -INFINITY;
        return;
    }
    const SampleTerms s = sample_terms(P, ray, flag);
    horizons[ray] = atan(s.slope) * (180.0 / M_PI);
}

static ScatterParams scatter_params(AdjointState &st, double *const *device_grads) {
    ScatterParams S{};
    S.checkpoints = st.checkpoints.as<float4>();
    S.flags = st.flags.as<uint8_t>();
    S.gradient = st.gradient.as<double>();
    for (size_t d = 0; d < st.dems.size(); ++d) {
        const ls200_dem *dem = st.dems[d];
        S.dems[d] = ScatterDem{dem->level0, device_grads ? device_grads[d] : nullptr, dem->width,
                               dem->height,
                               static_cast<double>(static_cast<float>(dem->projection[0]))};
    }
    for (int t = 0; t < st.tile_count; ++t) {
        S.origins[t] = st.origins[t];
        S.observer[t] = st.observer[t];
    }
    S.azimuth_count = st.azimuth_count;
    S.rays_per_tile = static_cast<long long>(kPatch) * kPatch * st.azimuth_count;
    S.total_rays = S.rays_per_tile * st.tile_count;
    return S;
}

static LossParams loss_params(AdjointState &st) {
    LossParams P{};
    P.horizons = st.horizons.as<float>();
    P.replayed = st.use_replayed ? st.replayed.as<double>() : nullptr;
    P.directions = st.directions.as<float2>();
    P.weights = st.weights.as<float>();
    P.gradient = st.gradient.as<double>();
    P.loss = st.loss.as<double>();
    for (int t = 0; t < st.tile_count; ++t) {
        const ls200_dem *primary = st.dems[0];
        P.valid[t] = make_int2(std::min(kPatch, primary->width - st.origins[t].x),
                               std::min(kPatch, primary->height - st.origins[t].y));
    }
    P.azimuth_count = st.azimuth_count;
    P.time_count = st.time_count;
    P.radius_deg = st.radius_deg;
    return P;
}

}  // namespace ls200

using namespace ls200;

extern "C" ls200_status ls200_sun_loss_forward(ls200_context *ctx, const ls200_site_tile *tiles,
                                               int tile_count, int azimuth_count, int traversal,
                                               const float *device_weights,
                                               const ls200_vectors *sun, double disk_radius_deg,
                                               double *loss, double *seconds) {
    return guard([&] {
        LS_REQUIRE(ctx && tiles && device_weights && sun && loss, "NULL argument");
        LS_REQUIRE(tile_count >= 1 && tile_count <= kMaxBatchTiles,
                   "1 to 32 tiles per adjoint problem");
        LS_REQUIRE(azimuth_count >= 4, "azimuth_count must be at least 4");
        LS_REQUIRE(traversal == 0 || traversal == 1, "the adjoint's traversal must be 0 or 1");
        LS_REQUIRE(disk_radius_deg > 0.0 && disk_radius_deg < 10.0,
                   "disk radius must be in (0, 10) degrees");
        LS_REQUIRE(sun->ctx == ctx && sun->count > 0, "sun vectors belong to another context");
        for (int t = 0; t < tile_count; ++t) {
            LS_REQUIRE(tiles[t].dem_count == tiles[0].dem_count && tiles[t].dem_count <= 8,
                       "every tile of an adjoint problem uses the same DEM stack");
            for (int d = 0; d < tiles[t].dem_count; ++d)
                LS_REQUIRE(tiles[t].dems[d] == tiles[0].dems[d],
                           "every tile of an adjoint problem uses the same DEM stack");
        }
        const size_t rays = static_cast<size_t>(tile_count) * kPatch * kPatch * azimuth_count;
        {
            std::lock_guard<std::mutex> hold(ctx->lock);
            activate(ctx);
            AdjointState &st = adjoint_of(ctx);
            st.ready = false;
            st.horizons.reserve(rays * sizeof(float));
            st.checkpoints.reserve(rays * sizeof(float4));
            st.flags.reserve(rays);
        }
        AdjointState &st = *ctx->adjoint;
        double march_seconds[2] = {0.0, 0.0};
        march_sites_run(ctx, tiles, tile_count, azimuth_count, 8, traversal, true,
                        st.horizons.as<float>(), march_seconds, st.checkpoints.as<float4>(),
                        st.flags.as<uint8_t>());
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        st.dems.assign(tiles[0].dems, tiles[0].dems + tiles[0].dem_count);
        st.origins.resize(tile_count);
        st.observer.resize(tile_count);
        for (int t = 0; t < tile_count; ++t) {
            st.origins[t] = make_int2(tiles[t].tile_column, tiles[t].tile_row);
            st.observer[t] = tiles[t].observer_elevation_m;
        }
        st.tile_count = tile_count;
        st.azimuth_count = azimuth_count;
        st.time_count = sun->count;
        st.radius_deg = disk_radius_deg;
        const size_t plane = static_cast<size_t>(kPatch) * kPatch;
        st.directions.reserve(sizeof(float2) * tile_count * plane * sun->count);
        st.patches.reserve(sizeof(float) * tile_count * plane + sizeof(int2) * tile_count);
        st.weights.reserve(sizeof(float) * tile_count * plane);
        st.loss.reserve(sizeof(double) * (1 + tile_count * plane / 128));
        ctx->scratch.reserve(sizeof(float) * 12 * tile_count * plane);
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[0], ctx->stream));
        LS_CUDA(cudaMemcpyAsync(st.weights.ptr, device_weights, sizeof(float) * tile_count * plane,
                                cudaMemcpyDeviceToDevice, ctx->stream));
        int2 *origins = reinterpret_cast<int2 *>(st.patches.as<float>() + tile_count * plane);
        LS_CUDA(cudaMemcpyAsync(origins, st.origins.data(), sizeof(int2) * tile_count,
                                cudaMemcpyHostToDevice, ctx->stream));
        const ls200_dem *primary = st.dems[0];
        gather_patches_kernel<<<dim3(plane / 128, tile_count), 128, 0, ctx->stream>>>(
            primary->level0, primary->width, primary->height, origins, st.patches.as<float>());
        LS_CUDA(cudaGetLastError());
        LightingBatch B{};
        for (int t = 0; t < tile_count; ++t) {
            std::memcpy(B.tiles[t].gt, primary->geo_transform, sizeof B.tiles[t].gt);
            std::memcpy(B.tiles[t].proj, primary->projection, sizeof B.tiles[t].proj);
            B.tiles[t].tile_x = st.origins[t].x;
            B.tiles[t].tile_y = st.origins[t].y;
            B.tiles[t].valid_width = std::min(kPatch, primary->width - st.origins[t].x);
            B.tiles[t].valid_height = std::min(kPatch, primary->height - st.origins[t].y);
        }
        B.patch_dem = st.patches.as<float>();
        B.vectors = sun->data;
        B.frames = ctx->scratch.as<float>();
        B.time_start = 0;
        B.time_count = sun->count;
        directions_launch(ctx, B, tile_count, st.directions.as<float2>());
        st.use_replayed = false;
        launch_loss(ctx, loss_params(st), tile_count);
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[1], ctx->stream));
        LS_CUDA(cudaMemcpyAsync(loss, st.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (seconds) {
            float ms = 0.0f;
            LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
            seconds[0] = march_seconds[0] + march_seconds[1];
            seconds[1] = ms / 1000.0;
        }
        st.ready = true;
    });
}

extern "C" ls200_status ls200_sun_loss_backward(ls200_context *ctx, double grad_output,
                                                double *const *device_grads, int grad_count,
                                                double *seconds) {
    return guard([&] {
        LS_REQUIRE(ctx && device_grads, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        LS_REQUIRE(ctx->adjoint && ctx->adjoint->ready, "no forward pass to differentiate");
        AdjointState &st = *ctx->adjoint;
        LS_REQUIRE(grad_count == static_cast<int>(st.dems.size()),
                   "one gradient array per DEM of the stack");
        for (int d = 0; d < grad_count; ++d) LS_REQUIRE(device_grads[d], "NULL gradient array");
        activate(ctx);
        const size_t rays =
            static_cast<size_t>(st.tile_count) * kPatch * kPatch * st.azimuth_count;
        st.gradient.reserve(rays * sizeof(double));
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[0], ctx->stream));
        LossParams P = loss_params(st);
        P.scale = grad_output / st.time_count;
        const size_t plane = static_cast<size_t>(kPatch) * kPatch;
        horizon_gradient_kernel<<<dim3(plane / 128, st.tile_count), 128, 0, ctx->stream>>>(P);
        LS_CUDA(cudaGetLastError());
        const ScatterParams S = scatter_params(st, device_grads);
        const unsigned blocks = static_cast<unsigned>((S.total_rays + 127) / 128);
        scatter_kernel<<<blocks, 128, 0, ctx->stream>>>(S);
        LS_CUDA(cudaGetLastError());
        if (seconds) LS_CUDA(cudaEventRecord(ctx->events[1], ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (seconds) {
            float ms = 0.0f;
            LS_CUDA(cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
            *seconds = ms / 1000.0;
        }
    });
}

extern "C" ls200_status ls200_sun_loss_replay(ls200_context *ctx, double *loss) {
    return guard([&] {
        LS_REQUIRE(ctx && loss, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        LS_REQUIRE(ctx->adjoint && ctx->adjoint->ready, "no forward pass to replay");
        AdjointState &st = *ctx->adjoint;
        activate(ctx);
        const ScatterParams S = scatter_params(st, nullptr);
        st.replayed.reserve(sizeof(double) * static_cast<size_t>(S.total_rays));
        replay_kernel<<<static_cast<unsigned>((S.total_rays + 127) / 128), 128, 0, ctx->stream>>>(
            S, st.replayed.as<double>());
        LS_CUDA(cudaGetLastError());
        st.use_replayed = true;
        launch_loss(ctx, loss_params(st), st.tile_count);
        LS_CUDA(cudaMemcpyAsync(loss, st.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" ls200_status ls200_sun_loss_checkpoints(ls200_context *ctx, float *points,
                                                   uint8_t *flags, float *directions,
                                                   float *horizons) {
    return guard([&] {
        LS_REQUIRE(ctx, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        LS_REQUIRE(ctx->adjoint && ctx->adjoint->ready, "no forward pass recorded");
        AdjointState &st = *ctx->adjoint;
        activate(ctx);
        const size_t rays =
            static_cast<size_t>(st.tile_count) * kPatch * kPatch * st.azimuth_count;
        const size_t dirs = static_cast<size_t>(st.tile_count) * st.time_count * kPatch * kPatch;
        if (points)
            LS_CUDA(cudaMemcpyAsync(points, st.checkpoints.ptr, rays * sizeof(float4),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        if (flags)
            LS_CUDA(cudaMemcpyAsync(flags, st.flags.ptr, rays, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        if (directions)
            LS_CUDA(cudaMemcpyAsync(directions, st.directions.ptr, dirs * sizeof(float2),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        if (horizons)
            LS_CUDA(cudaMemcpyAsync(horizons, st.horizons.ptr, rays * sizeof(float),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}
