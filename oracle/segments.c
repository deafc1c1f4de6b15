/*
 * ORACLE — test infrastructure only.  CPU restatement (FP64) of lunarscout's
 * host ray-segment generation: chord sampling against one DEM, the quartic
 * position fit and the planar->chord cubic fit.
 *
 * Follows src/lunarscout/_numba_horizon/geometry_numba.py:
 *   _solve        :30-64      Gauss-Jordan with partial pivoting
 *   _quartic      :67-91
 *   _chord_distance :94-100
 *   _fit_chord    :102-139
 *   _fit_one      :142-170
 *   _sample_chord :173-223
 *   _build_samples :226-295
 * Every expression keeps the reference's evaluation order; the build uses
 * -ffp-contract=off, and the transcendental calls are the same libm the
 * reference's Numba CPU code calls.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define NSAMP 16
#define NFIELD 8

typedef struct {
    const float *elevation;
    int width, height;
    const double *transform;  /* 6 */
    const double *projection; /* radius, lat0, lon0, scale, false_e, false_n */
} seg_dem;

static int sample_chord(const double obs[3], const double dir[3], double distance,
                        const seg_dem *dem, double out[NFIELD])
{
    const double *t = dem->transform, *p = dem->projection;
    double xv = obs[0] + dir[0] * distance;
    double yv = obs[1] + dir[1] * distance;
    double zv = obs[2] + dir[2] * distance;
    double longitude = atan2(yv, xv);
    if (longitude < 0.0) longitude += 2.0 * M_PI;
    double latitude = atan2(zv, sqrt(xv * xv + yv * yv));
    double sin_lat = sin(latitude), cos_lat = cos(latitude);
    double sin_o = sin(p[1]), cos_o = cos(p[1]);
    double delta = longitude - p[2];
    double denominator = 1.0 + sin_o * sin_lat + cos_o * cos_lat * cos(delta);
    if (fabs(denominator) < 1e-10) denominator = 1e-10;
    double scale = 2.0 * p[3] * p[0] / denominator;
    double px = scale * cos_lat * sin(delta) + p[4];
    double py = scale * (cos_o * sin_lat - sin_o * cos_lat * cos(delta)) + p[5];
    double det = t[1] * t[5] - t[2] * t[4];
    double dx = px - t[0], dy = py - t[3];
    double column = (t[5] * dx - t[2] * dy) / det;
    double row = (-t[4] * dx + t[1] * dy) / det;
    int inside = 0.0 <= column && column < dem->width && 0.0 <= row && row < dem->height;
    double terrain = 0.0;
    if (inside) {
        int x1 = (int)column, y1 = (int)row;
        int x2 = x1 + 1 < dem->width - 1 ? x1 + 1 : dem->width - 1;
        int y2 = y1 + 1 < dem->height - 1 ? y1 + 1 : dem->height - 1;
        const float *e = dem->elevation;
        size_t w = (size_t)dem->width;
        terrain = (double)e[y1 * w + x1] * (x2 - column) * (y2 - row) +
                  (double)e[y1 * w + x2] * (column - x1) * (y2 - row) +
                  (double)e[y2 * w + x1] * (x2 - column) * (row - y1) +
                  (double)e[y2 * w + x2] * (column - x1) * (row - y1);
    }
    out[0] = distance;
    out[1] = column;
    out[2] = row;
    out[3] = latitude;
    out[4] = longitude;
    out[5] = row;
    out[6] = column;
    out[7] = terrain;
    return inside;
}

static int build_samples(const double obs[3], const double dir[3], double start,
                         double maximum, const seg_dem *dem, double s[NSAMP][NFIELD])
{
    double first[NFIELD], end[NFIELD], sample[NFIELD], final_inside[NFIELD];
    memset(s, 0, sizeof(double) * NSAMP * NFIELD);
    if (!sample_chord(obs, dir, start, dem, first)) return 0;
    memcpy(s[0], first, sizeof first);
    int count = 1;
    memcpy(final_inside, first, sizeof first);
    if (sample_chord(obs, dir, maximum, dem, end)) {
        memcpy(final_inside, end, sizeof end);
    } else {
        double low = start, high = maximum;
        double best[NFIELD];
        memcpy(best, first, sizeof first);
        for (int i = 0; i < 24; ++i) {
            double middle = 0.5 * (low + high);
            if (sample_chord(obs, dir, middle, dem, sample)) {
                low = middle;
                memcpy(best, sample, sizeof sample);
            } else {
                high = middle;
            }
        }
        memcpy(final_inside, best, sizeof best);
    }
    double span = final_inside[0] - start;
    if (span < 0.0) span = 0.0;
    if (span > 1e-3) {
        for (int index = 1; index < 11; ++index) {
            double target = start + span * index / 10.0;
            if (target > final_inside[0] - 0.5) break;
            if (target - s[count - 1][0] < 0.5) continue;
            if (sample_chord(obs, dir, target, dem, sample)) {
                memcpy(s[count], sample, sizeof sample);
                ++count;
            }
        }
        if (count < NSAMP && final_inside[0] - s[count - 1][0] > 0.5) {
            memcpy(s[count], final_inside, sizeof final_inside);
            ++count;
        }
    }
    double required_end = s[0][0] + 100.0;
    const double *t = dem->transform;
    double map_resolution = 0.5 * (sqrt(t[1] * t[1] + t[4] * t[4]) +
                                   sqrt(t[2] * t[2] + t[5] * t[5]));
    if (count < 4 || s[count - 1][0] < required_end) {
        double step = map_resolution * 2.0 > 10.0 ? map_resolution * 2.0 : 10.0;
        double current = s[count - 1][0];
        double extend_limit = final_inside[0] > required_end ? final_inside[0] : required_end;
        while ((count < 4 || s[count - 1][0] < required_end) && current < extend_limit &&
               count < NSAMP) {
            current = extend_limit < current + step ? extend_limit : current + step;
            int inside = sample_chord(obs, dir, current, dem, sample);
            if (!inside || current - s[count - 1][0] < 0.5) break;
            memcpy(s[count], sample, sizeof sample);
            ++count;
        }
    }
    return count;
}

/* Gauss-Jordan elimination with partial pivoting on an n x (n+1) system. */
static int solve(int n, double a[4][5], double x[4])
{
    for (int index = 0; index < n; ++index) {
        int pivot = index;
        double maximum = fabs(a[index][index]);
        for (int row = index + 1; row < n; ++row) {
            double v = fabs(a[row][index]);
            if (v > maximum) {
                maximum = v;
                pivot = row;
            }
        }
        if (maximum < 1e-12) return 0;
        if (pivot != index) {
            for (int c = index; c <= n; ++c) {
                double v = a[index][c];
                a[index][c] = a[pivot][c];
                a[pivot][c] = v;
            }
        }
        double divisor = a[index][index];
        for (int c = index; c <= n; ++c) a[index][c] /= divisor;
        for (int row = 0; row < n; ++row) {
            if (row == index) continue;
            double factor = a[row][index];
            if (fabs(factor) < 1e-12) continue;
            for (int c = index; c <= n; ++c) a[row][c] -= factor * a[index][c];
        }
    }
    for (int r = 0; r < n; ++r) x[r] = a[r][n];
    return 1;
}

static void quartic(double s[NSAMP][NFIELD], int count, int column, double value0,
                    double anchor_km, double span_km, double out[4])
{
    double a[4][5];
    memset(a, 0, sizeof a);
    for (int i = 0; i < count; ++i) {
        double parameter = (s[i][0] / 1000.0 - anchor_km) / span_km;
        double powers[4];
        powers[0] = parameter;
        for (int k = 1; k < 4; ++k) powers[k] = powers[k - 1] * parameter;
        double value = s[i][column] - value0;
        for (int r = 0; r < 4; ++r) {
            a[r][4] += powers[r] * value;
            for (int c = 0; c < 4; ++c) a[r][c] += powers[r] * powers[c];
        }
    }
    double x[4];
    if (!solve(4, a, x)) {
        out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    double inverse = 1.0 / span_km, scale = inverse;
    for (int k = 0; k < 4; ++k) {
        out[k] = x[k] * scale;
        scale *= inverse;
    }
}

static double chord_distance(const double obs[3], double latitude, double longitude,
                             double radius)
{
    double cos_latitude = cos(latitude);
    double x = radius * cos_latitude * cos(longitude) - obs[0];
    double y = radius * cos_latitude * sin(longitude) - obs[1];
    double z = radius * sin(latitude) - obs[2];
    return sqrt(x * x + y * y + z * z);
}

static void fit_chord(double s[NSAMP][NFIELD], int count, double map_resolution,
                      const double obs[3], double radius, double out[3])
{
    out[0] = 1.0;
    out[1] = 0.0;
    out[2] = 0.0;
    if (count < 2 || map_resolution <= 0.0) return;
    double planar[NSAMP] = {0}, chord[NSAMP] = {0};
    double chord0 = chord_distance(obs, s[0][3], s[0][4], radius);
    double maximum_planar = 0.0;
    int used = 1;
    int limit = count < NSAMP ? count : NSAMP;
    for (int i = 1; i < limit; ++i) {
        if (s[i][1] < 0.0 || s[i][2] < 0.0) continue;
        double dx = (s[i][1] - s[0][1]) * map_resolution;
        double dy = (s[i][2] - s[0][2]) * map_resolution;
        double distance = sqrt(dx * dx + dy * dy);
        planar[used] = distance;
        chord[used] = chord_distance(obs, s[i][3], s[i][4], radius) - chord0;
        if (distance > maximum_planar) maximum_planar = distance;
        ++used;
    }
    if (used < 2 || maximum_planar < 500.0) return;
    double a[4][5];
    memset(a, 0, sizeof a);
    for (int i = 0; i < used; ++i) {
        double x = planar[i];
        double powers[3] = {x, x * x, x * x * x};
        for (int r = 0; r < 3; ++r) {
            a[r][3] += powers[r] * chord[i];
            for (int c = 0; c < 3; ++c) a[r][c] += powers[r] * powers[c];
        }
    }
    /* solve() expects the right-hand side in column n. */
    double b[4][5];
    memset(b, 0, sizeof b);
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) b[r][c] = a[r][c];
        b[r][3] = a[r][3];
    }
    double x[4];
    if (!solve(3, b, x) || x[0] < 0.5 || x[0] > 2.0) return;
    out[0] = x[0];
    out[1] = x[1];
    out[2] = x[2];
}

static void fit_one(double s[NSAMP][NFIELD], int count, double map_resolution,
                    const double obs[3], double radius, double fallback_start,
                    float out[18])
{
    memset(out, 0, sizeof(float) * 18);
    if (count < 3) {
        double x = count ? s[0][1] : 0.0;
        double y = count ? s[0][2] : 0.0;
        double start = count ? s[0][0] / 1000.0 : fallback_start / 1000.0;
        out[0] = (float)x;
        out[1] = (float)y;
        out[2] = (float)x;
        out[3] = (float)y;
        out[12] = (float)start;
        out[13] = (float)start;
        out[14] = (float)start;
        out[15] = 1.0f;
        return;
    }
    double x0 = s[0][1], y0 = s[0][2];
    double anchor_km = s[0][0] / 1000.0;
    double end_km = s[count - 1][0] / 1000.0;
    double span_km = end_km - anchor_km;
    if (span_km < 0.001) span_km = 0.001;
    double xc[4], yc[4], ch[3];
    quartic(s, count, 1, x0, anchor_km, span_km, xc);
    quartic(s, count, 2, y0, anchor_km, span_km, yc);
    fit_chord(s, count, map_resolution, obs, radius, ch);
    out[0] = (float)x0;
    out[1] = (float)y0;
    out[2] = (float)x0;
    out[3] = (float)y0;
    for (int k = 0; k < 4; ++k) {
        out[4 + k] = (float)xc[k];
        out[8 + k] = (float)yc[k];
    }
    out[12] = (float)anchor_km;
    out[13] = (float)end_km;
    out[14] = (float)anchor_km;
    out[15] = (float)ch[0];
    out[16] = (float)ch[1];
    out[17] = (float)ch[2];
}

/* generate_segments_parallel (geometry_numba.py:352-364) for one DEM:
 * observers/directions [n,3], starts/radii [n]; `maximum` is the DEM's ray
 * limit; writes out [n,18]. */
int ora_segments_dem(const float *elevation, int width, int height,
                     const double *transform, const double *projection,
                     const double *observers, const double *directions,
                     const double *starts, double maximum, double map_resolution,
                     const double *radii, long long n, float *out, int threads)
{
    seg_dem dem = {elevation, width, height, transform, projection};
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 32) num_threads(threads)
    for (long long i = 0; i < n; ++i) {
        double samples[NSAMP][NFIELD];
        int count = build_samples(observers + 3 * i, directions + 3 * i, starts[i], maximum,
                                  &dem, samples);
        fit_one(samples, count, map_resolution, observers + 3 * i, radii[i], starts[i],
                out + 18 * i);
    }
    return 0;
}

/* The chord samples of one job, for inspection: returns the count and writes
 * [16, 8] rows. */
int ora_segment_samples(const float *elevation, int width, int height,
                        const double *transform, const double *projection,
                        const double *observer, const double *direction, double start,
                        double maximum, double *rows)
{
    seg_dem dem = {elevation, width, height, transform, projection};
    double samples[NSAMP][NFIELD];
    int count = build_samples(observer, direction, start, maximum, &dem, samples);
    memcpy(rows, samples, sizeof samples);
    return count;
}
