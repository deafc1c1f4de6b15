// Ray-segment generation on the device (FP64): for every subpatch centre and
// azimuth of a tile, sample the Moon-centred ray chord against one DEM and
// fit the quartic pixel path and the planar->chord cubic the march consumes.
//
// Semantics follow src/lunarscout/_numba_horizon/geometry.py:575-673
// (build_subpatch_segments_numba: centres, observers, directions, the
// cross-DEM start carry) and geometry_numba.py:30-364 (sampling and fits).
// The reference does this on the host with Numba at ~2 s per 4-DEM tile;
// here one thread owns one (centre, azimuth) job of one DEM.  FP64 is used
// throughout, as in the reference; the stored fields are float32.
#include "internal.cuh"

namespace ls200 {

namespace {

constexpr int kSamples = 16;

struct SegDem {
    const float *elevation;
    int width, height;
    double t[6];  // geo transform
    double p[6];  // projection
    double resolution;   // (hypot(t1,t4) + hypot(t2,t5)) / 2
    double sample_resolution;  // the same with sqrt(x*x + y*y)
    double ray_limit;
};

struct SegParams {
    SegDem primary;
    SegDem dem;
    int dem_index, dem_count;
    int tile_column, tile_row, tile_width, subpatch, azimuth_count, center_count;
    double maximum_distance, observer_elevation;
    double *starts;  // [A*C] carried start distance (m)
    float *segments; // [A, C, D, 18]
};

struct Sample {
    double distance, column, row, latitude, longitude;
};

__device__ bool sample_chord(const double obs[3], const double dir[3], double distance,
                             const SegDem &dem, Sample &out) {
    const double *t = dem.t, *p = dem.p;
    const double xv = obs[0] + dir[0] * distance;
    const double yv = obs[1] + dir[1] * distance;
    const double zv = obs[2] + dir[2] * distance;
    double longitude = atan2(yv, xv);
    if (longitude < 0.0) longitude += 2.0 * 3.141592653589793;
    const double latitude = atan2(zv, sqrt(xv * xv + yv * yv));
    double sin_lat, cos_lat;
    sincos(latitude, &sin_lat, &cos_lat);
    double sin_o, cos_o;
    sincos(p[1], &sin_o, &cos_o);
    const double delta = longitude - p[2];
    double sin_d, cos_d;
    sincos(delta, &sin_d, &cos_d);
    double denominator = 1.0 + sin_o * sin_lat + cos_o * cos_lat * cos_d;
    if (fabs(denominator) < 1e-10) denominator = 1e-10;
    const double scale = 2.0 * p[3] * p[0] / denominator;
    const double px = scale * cos_lat * sin_d + p[4];
    const double py = scale * (cos_o * sin_lat - sin_o * cos_lat * cos_d) + p[5];
    const double det = t[1] * t[5] - t[2] * t[4];
    const double dx = px - t[0], dy = py - t[3];
    const double column = (t[5] * dx - t[2] * dy) / det;
    const double row = (-t[4] * dx + t[1] * dy) / det;
    out.distance = distance;
    out.column = column;
    out.row = row;
    out.latitude = latitude;
    out.longitude = longitude;
    return 0.0 <= column && column < dem.width && 0.0 <= row && row < dem.height;
}

__device__ int build_samples(const double obs[3], const double dir[3], double start,
                             double maximum, const SegDem &dem, Sample *s) {
    Sample first, sample, final_inside;
    if (!sample_chord(obs, dir, start, dem, first)) return 0;
    s[0] = first;
    int count = 1;
    final_inside = first;
    if (sample_chord(obs, dir, maximum, dem, sample)) {
        final_inside = sample;
    } else {
        double low = start, high = maximum;
        Sample best = first;
        for (int i = 0; i < 24; ++i) {
            const double middle = 0.5 * (low + high);
            if (sample_chord(obs, dir, middle, dem, sample)) {
                low = middle;
                best = sample;
            } else {
                high = middle;
            }
        }
        final_inside = best;
    }
    double span = final_inside.distance - start;
    if (span < 0.0) span = 0.0;
    if (span > 1e-3) {
        for (int index = 1; index < 11; ++index) {
            const double target = start + span * index / 10.0;
            if (target > final_inside.distance - 0.5) break;
            if (target - s[count - 1].distance < 0.5) continue;
            if (sample_chord(obs, dir, target, dem, sample)) s[count++] = sample;
        }
        if (count < kSamples && final_inside.distance - s[count - 1].distance > 0.5)
            s[count++] = final_inside;
    }
    const double required_end = s[0].distance + 100.0;
    if (count < 4 || s[count - 1].distance < required_end) {
        const double step = dem.sample_resolution * 2.0 > 10.0 ? dem.sample_resolution * 2.0 : 10.0;
        double current = s[count - 1].distance;
        const double extend_limit =
            final_inside.distance > required_end ? final_inside.distance : required_end;
        while ((count < 4 || s[count - 1].distance < required_end) && current < extend_limit &&
               count < kSamples) {
            current = extend_limit < current + step ? extend_limit : current + step;
            const bool inside = sample_chord(obs, dir, current, dem, sample);
            if (!inside || current - s[count - 1].distance < 0.5) break;
            s[count++] = sample;
        }
    }
    return count;
}

// Gauss-Jordan with partial pivoting on an n x (n+1) augmented system.
template <int N>
__device__ bool solve(double a[N][N + 1], double x[N]) {
    for (int index = 0; index < N; ++index) {
        int pivot = index;
        double maximum = fabs(a[index][index]);
        for (int row = index + 1; row < N; ++row) {
            const double v = fabs(a[row][index]);
            if (v > maximum) {
                maximum = v;
                pivot = row;
            }
        }
        if (maximum < 1e-12) return false;
        if (pivot != index) {
            for (int c = index; c <= N; ++c) {
                const double v = a[index][c];
                a[index][c] = a[pivot][c];
                a[pivot][c] = v;
            }
        }
        const double divisor = a[index][index];
        for (int c = index; c <= N; ++c) a[index][c] /= divisor;
        for (int row = 0; row < N; ++row) {
            if (row == index) continue;
            const double factor = a[row][index];
            if (fabs(factor) < 1e-12) continue;
            for (int c = index; c <= N; ++c) a[row][c] -= factor * a[index][c];
        }
    }
    for (int r = 0; r < N; ++r) x[r] = a[r][N];
    return true;
}

__device__ void fit_quartic(const Sample *s, int count, bool use_row, double value0,
                            double anchor_km, double span_km, double out[4]) {
    double a[4][5] = {};
    for (int i = 0; i < count; ++i) {
        const double parameter = (s[i].distance / 1000.0 - anchor_km) / span_km;
        double powers[4];
        powers[0] = parameter;
        for (int k = 1; k < 4; ++k) powers[k] = powers[k - 1] * parameter;
        const double value = (use_row ? s[i].row : s[i].column) - value0;
        for (int r = 0; r < 4; ++r) {
            a[r][4] += powers[r] * value;
            for (int c = 0; c < 4; ++c) a[r][c] += powers[r] * powers[c];
        }
    }
    double x[4];
    if (!solve<4>(a, x)) {
        out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    const double inverse = 1.0 / span_km;
    double scale = inverse;
    for (int k = 0; k < 4; ++k) {
        out[k] = x[k] * scale;
        scale *= inverse;
    }
}

__device__ double chord_distance(const double obs[3], double latitude, double longitude,
                                 double radius) {
    double sin_lat, cos_lat, sin_lon, cos_lon;
    sincos(latitude, &sin_lat, &cos_lat);
    sincos(longitude, &sin_lon, &cos_lon);
    const double x = radius * cos_lat * cos_lon - obs[0];
    const double y = radius * cos_lat * sin_lon - obs[1];
    const double z = radius * sin_lat - obs[2];
    return sqrt(x * x + y * y + z * z);
}

__device__ void fit_chord(const Sample *s, int count, double map_resolution,
                          const double obs[3], double radius, double out[3]) {
    out[0] = 1.0;
    out[1] = 0.0;
    out[2] = 0.0;
    if (count < 2 || map_resolution <= 0.0) return;
    double planar[kSamples], chord[kSamples];
    planar[0] = 0.0;
    chord[0] = 0.0;
    const double chord0 = chord_distance(obs, s[0].latitude, s[0].longitude, radius);
    double maximum_planar = 0.0;
    int used = 1;
    const int limit = count < kSamples ? count : kSamples;
    for (int i = 1; i < limit; ++i) {
        if (s[i].column < 0.0 || s[i].row < 0.0) continue;
        const double dx = (s[i].column - s[0].column) * map_resolution;
        const double dy = (s[i].row - s[0].row) * map_resolution;
        const double distance = sqrt(dx * dx + dy * dy);
        planar[used] = distance;
        chord[used] = chord_distance(obs, s[i].latitude, s[i].longitude, radius) - chord0;
        if (distance > maximum_planar) maximum_planar = distance;
        ++used;
    }
    if (used < 2 || maximum_planar < 500.0) return;
    double a[3][4] = {};
    for (int i = 0; i < used; ++i) {
        const double x = planar[i];
        const double powers[3] = {x, x * x, x * x * x};
        for (int r = 0; r < 3; ++r) {
            a[r][3] += powers[r] * chord[i];
            for (int c = 0; c < 3; ++c) a[r][c] += powers[r] * powers[c];
        }
    }
    double x[3];
    if (!solve<3>(a, x) || x[0] < 0.5 || x[0] > 2.0) return;
    out[0] = x[0];
    out[1] = x[1];
    out[2] = x[2];
}

__device__ int clamp_center(int requested, int dem_size, int subpatch) {
    const int half = subpatch / 2;
    const int upper = dem_size - half > half ? dem_size - half : half;
    return requested < half ? half : (requested > upper ? upper : requested);
}

// DemGrid.elevation (geometry.py:98-110): FP64 bilinear without validity.
__device__ double dem_elevation(const SegDem &dem, double column, double row) {
    const int x1 = static_cast<int>(column), y1 = static_cast<int>(row);
    const int x2 = min(x1 + 1, dem.width - 1), y2 = min(y1 + 1, dem.height - 1);
    const float *e = dem.elevation;
    const size_t w = static_cast<size_t>(dem.width);
    return static_cast<double>(e[y1 * w + x1]) * (x2 - column) * (y2 - row) +
           static_cast<double>(e[y1 * w + x2]) * (column - x1) * (y2 - row) +
           static_cast<double>(e[y2 * w + x1]) * (x2 - column) * (row - y1) +
           static_cast<double>(e[y2 * w + x2]) * (column - x1) * (row - y1);
}

__global__ void __launch_bounds__(128) segments_kernel(const __grid_constant__ SegParams P) {
    const int job = blockIdx.x * blockDim.x + threadIdx.x;
    if (job >= P.azimuth_count * P.center_count) return;
    // Job order: azimuth fastest within a centre keeps one centre's setup
    // in neighbouring threads.
    const int center = job / P.azimuth_count;
    const int azimuth = job % P.azimuth_count;
    const double start = P.dem_index == 0 ? 1.0 : P.starts[job];
    if (!(start < P.maximum_distance)) return;  // finished in an earlier DEM

    // ---- centre geometry (geometry.py:613-634) ----
    const SegDem &pri = P.primary;
    const int count = P.tile_width / P.subpatch + 2;
    const int grid_row = center / count, grid_column = center % count;
    const int cc = clamp_center(P.tile_column + (grid_column - 1) * P.subpatch + P.subpatch / 2,
                                pri.width, P.subpatch);
    const int cr = clamp_center(P.tile_row + (grid_row - 1) * P.subpatch + P.subpatch / 2,
                                pri.height, P.subpatch);
    const double x = pri.t[0] + pri.t[1] * cc + pri.t[2] * cr;
    const double y = pri.t[3] + pri.t[4] * cc + pri.t[5] * cr;
    const double xp = x - pri.p[4], yp = y - pri.p[5];
    const double rho = hypot(xp, yp);
    double latitude = pri.p[1], longitude = pri.p[2];
    if (!(rho < 1e-9)) {
        const double c = 2.0 * atan2(rho, 2.0 * pri.p[3] * pri.p[0]);
        double sin_c, cos_c, sin_o, cos_o;
        sincos(c, &sin_c, &cos_c);
        sincos(pri.p[1], &sin_o, &cos_o);
        latitude = asin(cos_c * sin_o + yp * sin_c * cos_o / rho);
        longitude = pri.p[2] + atan2(xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c);
    }
    const double tc = fmin(fmax(static_cast<double>(cc), 0.0), pri.width - 1.001);
    const double tr = fmin(fmax(static_cast<double>(cr), 0.0), pri.height - 1.001);
    const double radius = pri.p[0] + dem_elevation(pri, tc, tr);
    const double r = radius + P.observer_elevation;
    double sin_lat, cos_lat, sin_lon, cos_lon;
    sincos(latitude, &sin_lat, &cos_lat);
    sincos(longitude, &sin_lon, &cos_lon);
    const double obs[3] = {r * cos_lat * cos_lon, r * cos_lat * sin_lon, r * sin_lat};
    const double angle = 3.141592653589793 / 2.0 -
                         azimuth * 2.0 * 3.141592653589793 / P.azimuth_count;
    double sa, ca;
    sincos(angle, &sa, &ca);
    double dir[3] = {ca * -sin_lon + sa * (-sin_lat * cos_lon),
                     ca * cos_lon + sa * (-sin_lat * sin_lon), sa * cos_lat};
    const double norm = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    dir[0] /= norm;
    dir[1] /= norm;
    dir[2] /= norm;

    // ---- sample and fit (geometry_numba.py:142-170, 226-295) ----
    Sample s[kSamples];
    const int n = build_samples(obs, dir, start, P.dem.ray_limit, P.dem, s);
    float out[kSegmentFields] = {};
    if (n < 3) {
        const double sx = n ? s[0].column : 0.0, sy = n ? s[0].row : 0.0;
        const double st = n ? s[0].distance / 1000.0 : start / 1000.0;
        out[0] = out[2] = static_cast<float>(sx);
        out[1] = out[3] = static_cast<float>(sy);
        out[12] = out[13] = out[14] = static_cast<float>(st);
        out[15] = 1.0f;
    } else {
        const double x0 = s[0].column, y0 = s[0].row;
        const double anchor_km = s[0].distance / 1000.0;
        const double end_km = s[n - 1].distance / 1000.0;
        const double span_km = end_km - anchor_km < 0.001 ? 0.001 : end_km - anchor_km;
        double xc[4], yc[4], ch[3];
        fit_quartic(s, n, false, x0, anchor_km, span_km, xc);
        fit_quartic(s, n, true, y0, anchor_km, span_km, yc);
        fit_chord(s, n, P.dem.resolution, obs, radius, ch);
        out[0] = out[2] = static_cast<float>(x0);
        out[1] = out[3] = static_cast<float>(y0);
        for (int k = 0; k < 4; ++k) {
            out[4 + k] = static_cast<float>(xc[k]);
            out[8 + k] = static_cast<float>(yc[k]);
        }
        out[12] = out[14] = static_cast<float>(anchor_km);
        out[13] = static_cast<float>(end_km);
        out[15] = static_cast<float>(ch[0]);
        out[16] = static_cast<float>(ch[1]);
        out[17] = static_cast<float>(ch[2]);
    }
    float *dst = P.segments +
                 ((static_cast<size_t>(azimuth) * P.center_count + center) * P.dem_count +
                  P.dem_index) * kSegmentFields;
#pragma unroll
    for (int k = 0; k < kSegmentFields; ++k) dst[k] = out[k];
    // The next DEM starts where this one's fit ended (float32 end, in m).
    const double last = static_cast<double>(out[13]) * 1000.0;
    P.starts[job] = P.dem.ray_limit < last ? P.dem.ray_limit : last;
}

SegDem make_dem(const ls200_dem *d, double maximum_distance) {
    SegDem s{};
    s.elevation = d->level0;
    s.width = d->width;
    s.height = d->height;
    std::memcpy(s.t, d->geo_transform, sizeof s.t);
    std::memcpy(s.p, d->projection, sizeof s.p);
    s.resolution = (std::hypot(s.t[1], s.t[4]) + std::hypot(s.t[2], s.t[5])) * 0.5;
    s.sample_resolution = 0.5 * (std::sqrt(s.t[1] * s.t[1] + s.t[4] * s.t[4]) +
                                 std::sqrt(s.t[2] * s.t[2] + s.t[5] * s.t[5]));
    const double size_m = std::min(s.width * s.resolution, s.height * s.resolution);
    s.ray_limit = std::min(maximum_distance, size_m * 1.2);
    return s;
}

}  // namespace

void segments_device(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                     int tile_column, int tile_row, int tile_width, int azimuth_count,
                     double maximum_distance_m, double observer_elevation_m, int subpatch,
                     float *device_segments) {
    const int count = tile_width / subpatch + 2;
    const int centers = count * count;
    const int jobs = centers * azimuth_count;
    ctx->scratch.reserve(sizeof(double) * size_t(jobs));
    LS_CUDA(cudaMemsetAsync(device_segments, 0,
                            sizeof(float) * size_t(jobs) * dem_count * kSegmentFields,
                            ctx->stream));
    SegParams P{};
    P.primary = make_dem(dems[0], maximum_distance_m);
    P.dem_count = dem_count;
    P.tile_column = tile_column;
    P.tile_row = tile_row;
    P.tile_width = tile_width;
    P.subpatch = subpatch;
    P.azimuth_count = azimuth_count;
    P.center_count = centers;
    P.maximum_distance = maximum_distance_m;
    P.observer_elevation = observer_elevation_m;
    P.starts = ctx->scratch.as<double>();
    P.segments = device_segments;
    for (int d = 0; d < dem_count; ++d) {
        P.dem = make_dem(dems[d], maximum_distance_m);
        // A segment ends within the DEM's ray limit (the path is at most a
        // few percent longer than the chord).
        require_march_progress(P.dem.ray_limit * 1.05e-3 + 1.0, dems[d]);
        P.dem_index = d;
        segments_kernel<<<(jobs + 127) / 128, 128, 0, ctx->stream>>>(P);
        LS_CUDA(cudaGetLastError());
    }
}

}  // namespace ls200

using namespace ls200;

extern "C" {

ls200_status ls200_segments_device(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                                   int tile_column, int tile_row, int tile_width,
                                   int azimuth_count, double maximum_distance_m,
                                   double observer_elevation_m, int subpatch_size,
                                   float *device_segments) {
    return guard([&] {
        LS_REQUIRE(ctx && dems && device_segments && dem_count > 0, "NULL argument");
        LS_REQUIRE(azimuth_count > 0 && tile_width > 0 && subpatch_size > 0,
                   "segment dimensions must be positive");
        LS_REQUIRE(maximum_distance_m > 0.0, "maximum_distance_m must be positive");
        for (int d = 0; d < dem_count; ++d) LS_REQUIRE(dems[d] != nullptr, "NULL DEM");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        segments_device(ctx, dems, dem_count, tile_column, tile_row, tile_width, azimuth_count,
                        maximum_distance_m, observer_elevation_m, subpatch_size,
                        device_segments);
    });
}

ls200_status ls200_segments(ls200_context *ctx, ls200_dem *const *dems, int dem_count,
                            int tile_column, int tile_row, int tile_width, int azimuth_count,
                            double maximum_distance_m, double observer_elevation_m,
                            int subpatch_size, float *segments) {
    return guard([&] {
        LS_REQUIRE(ctx && dems && segments && dem_count > 0, "NULL argument");
        LS_REQUIRE(azimuth_count > 0 && tile_width > 0 && subpatch_size > 0,
                   "segment dimensions must be positive");
        LS_REQUIRE(maximum_distance_m > 0.0, "maximum_distance_m must be positive");
        for (int d = 0; d < dem_count; ++d) LS_REQUIRE(dems[d] != nullptr, "NULL DEM");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        const int count = tile_width / subpatch_size + 2;
        const size_t bytes = sizeof(float) * size_t(azimuth_count) * count * count * dem_count *
                             kSegmentFields;
        ctx->segments.reserve(bytes);
        segments_device(ctx, dems, dem_count, tile_column, tile_row, tile_width, azimuth_count,
                        maximum_distance_m, observer_elevation_m, subpatch_size,
                        ctx->segments.as<float>());
        LS_CUDA(cudaMemcpyAsync(segments, ctx->segments.ptr, bytes, cudaMemcpyDeviceToHost,
                                ctx->stream));
        LS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
