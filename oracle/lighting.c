/*
 * ORACLE — test infrastructure only.  CPU restatement of lunarscout's
 * per-pixel lighting products against a 1440-azimuth horizon tile.
 *
 * lighting_frame / lighting_tile follow
 *   src/lunarscout/_numba_horizon/lightmap_cpu.py:25-183 (the "cpu" backend:
 *   FP64 east/north/up frame per pixel, float32 per time step, sun fraction
 *   over 16 half-disk slices, or body-centre margin), with the constants of
 *   src/lunarscout/_numba_horizon/lightmap.py:15-29.
 * psr_tile follows src/lunarscout/_numba_horizon/psr.py:29-58, 94-140
 *   (compute_psr_patch_reference: FP64 throughout, upper-limb threshold
 *   -0.545/2 deg).
 * Expressions keep the reference's order; the build uses -ffp-contract=off.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define AZ 1440
#define PATCH 128

/* float32 half-disk heights of the 16 slices (lightmap.py:19-25): the
 * half-chord of a 16-column discretised disk of radius 0.27 deg. */
static void half_circle(float out[16])
{
    for (int i = 0; i < 16; ++i) {
        double x = 7.5 - i;
        out[i] = (float)(sqrt(64.0 - x * x) / 8.0 * (double)0.27f);
    }
}

static float max_photons(const float hc[16])
{
    float sum = 0.0f;
    for (int i = 0; i < 16; ++i) sum = sum + hc[i];
    return 2.0f * sum;
}

typedef struct {
    float r00, r01, r02, r10, r11, r12, r20, r21, r22, tx, ty, tz;
} frame32;

/* FP64 frame of one DEM pixel (lightmap_cpu.py:51-103). */
static frame32 pixel_frame(const double *gt, const double *proj, int column, int row,
                           float height)
{
    double crs_x = gt[0] + gt[1] * column + gt[2] * row;
    double crs_y = gt[3] + gt[4] * column + gt[5] * row;
    double xp = crs_x - proj[4];
    double yp = crs_y - proj[5];
    double rho = sqrt(xp * xp + yp * yp);
    double latitude, longitude;
    if (rho <= 1e-12) {
        longitude = proj[2];
        latitude = proj[1];
    } else {
        double c = 2.0 * atan2(rho, 2.0 * proj[3] * proj[0]);
        double sin_c = sin(c), cos_c = cos(c);
        double cos_o = cos(proj[1]), sin_o = sin(proj[1]);
        latitude = asin(cos_c * sin_o + yp * sin_c * cos_o / rho);
        longitude = proj[2] + atan2(xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c);
    }
    double radius = proj[0] + (double)height;
    double cos_lat = cos(latitude), sin_lat = sin(latitude);
    double cos_lon = cos(longitude), sin_lon = sin(longitude);
    double moon_x = radius * cos_lat * cos_lon;
    double moon_y = radius * cos_lat * sin_lon;
    double moon_z = radius * sin_lat;
    double up_x = cos_lat * cos_lon, up_y = cos_lat * sin_lon, up_z = sin_lat;
    double east_x = -sin_lon, east_y = cos_lon;
    double north_x = -sin_lat * cos_lon, north_y = -sin_lat * sin_lon, north_z = cos_lat;
    frame32 f;
    f.tx = (float)(-(moon_x * east_x + moon_y * east_y));
    f.ty = (float)(-(moon_x * north_x + moon_y * north_y + moon_z * north_z));
    f.tz = (float)(-(moon_x * up_x + moon_y * up_y + moon_z * up_z));
    f.r00 = (float)east_x;
    f.r01 = (float)north_x;
    f.r02 = (float)up_x;
    f.r10 = (float)east_y;
    f.r11 = (float)north_y;
    f.r12 = (float)up_y;
    f.r20 = 0.0f;
    f.r21 = (float)north_z;
    f.r22 = (float)up_z;
    return f;
}

static const float DEG = 57.29577951308232f;

/* Sun fraction (or body-centre margin when `margin`) of one pixel and one
 * float32 Moon-ME vector (lightmap_cpu.py:105-183). */
static float pixel_signal(const frame32 *f, const float *v, const float *horizon, int margin,
                          const float hc[16], float photons_max)
{
    float vx = v[0], vy = v[1], vz = v[2];
    float enu_x = vx * f->r00 + vy * f->r10 + vz * f->r20 + f->tx;
    float enu_y = vx * f->r01 + vy * f->r11 + vz * f->r21 + f->ty;
    float enu_z = vx * f->r02 + vy * f->r12 + vz * f->r22 + f->tz;
    float horizontal = sqrtf(enu_x * enu_x + enu_y * enu_y);
    float elevation = atan2f(enu_z, horizontal) * DEG;
    float azimuth = atan2f(enu_x, enu_y);
    if (azimuth < 0.0f) azimuth = azimuth + (float)(M_PI * 2.0);
    float azimuth_deg = azimuth * DEG;
    if (margin) {
        float center_position = azimuth_deg * 4.0f;
        int left = (int)center_position;
        float fraction = center_position - (float)left;
        if (left >= AZ) left -= AZ;
        int right = left + 1;
        if (right >= AZ) right = 0;
        float h = horizon[left] + fraction * (horizon[right] - horizon[left]);
        return elevation - h;
    }
    float left_position = (azimuth_deg - 0.27f - 0.125f) * 4.0f;
    int left = (int)left_position;
    float fraction = left_position - (float)left;
    if (left < 0) left += AZ;
    else if (left >= AZ) left -= AZ;
    int right = left + 1;
    if (right >= AZ) right = 0;
    float left_elevation = horizon[left];
    float right_elevation = horizon[right];
    float delta = right_elevation - left_elevation;
    float photons = 0.0f;
    for (int s = 0; s < 16; ++s) {
        float h = fraction * delta + left_elevation;
        float column = hc[s];
        float sun_top = elevation + column;
        if (h < sun_top) {
            float angle_delta = sun_top - h;
            float column_height = column + column;
            if (angle_delta > column_height) angle_delta = column_height;
            photons = photons + angle_delta;
        }
        fraction = fraction + 0.135f;
        if (fraction >= 1.0f) {
            left = right;
            right += 1;
            if (right >= AZ) right = 0;
            left_elevation = right_elevation;
            right_elevation = horizon[right];
            delta = right_elevation - left_elevation;
            fraction = fraction - 1.0f;
        }
    }
    return photons / photons_max;
}

/* One tile: patch_dem float32[128,128] (zero outside the valid rect),
 * horizons float32[128,128,1440] degrees, vectors float32[T,3];
 * out float32[T,128,128] (zeros outside the valid rect). */
int ora_lighting_tile(const float *patch_dem, const double *gt, const double *proj,
                      const float *vectors, int count, const float *horizons, int tile_x,
                      int tile_y, int valid_width, int valid_height, int margin, float *out,
                      int threads)
{
    float hc[16];
    half_circle(hc);
    float pm = max_photons(hc);
    if (threads < 1) threads = 1;
    memset(out, 0, sizeof(float) * (size_t)count * PATCH * PATCH);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int index = 0; index < PATCH * PATCH; ++index) {
        int sample = index % PATCH, line = index / PATCH;
        if (sample >= valid_width || line >= valid_height) continue;
        frame32 f = pixel_frame(gt, proj, tile_x + sample, tile_y + line,
                                patch_dem[line * PATCH + sample]);
        const float *h = horizons + (size_t)index * AZ;
        for (int t = 0; t < count; ++t)
            out[(size_t)t * PATCH * PATCH + index] =
                pixel_signal(&f, vectors + 3 * (size_t)t, h, margin, hc, pm);
    }
    return 0;
}

/* Sun fraction at a given float32 azimuth/elevation (deg) over n horizon
 * rows (lightmap.py:32-73, the C# BuilderSunFraction). */
int ora_sun_fraction(const float *horizons, const float *azimuth_deg, const float *elevation,
                     int n, float *out)
{
    float hc[16];
    half_circle(hc);
    float pm = max_photons(hc);
    for (int i = 0; i < n; ++i) {
        const float *horizon = horizons + (size_t)i * AZ;
        float left_position = (azimuth_deg[i] - 0.27f - 0.125f) * 4.0f;
        int left = (int)left_position;
        float fraction = left_position - (float)left;
        if (left < 0) left += AZ;
        else if (left >= AZ) left -= AZ;
        int right = left + 1;
        if (right >= AZ) right = 0;
        float left_elevation = horizon[left], right_elevation = horizon[right];
        float delta = right_elevation - left_elevation;
        float photons = 0.0f;
        for (int s = 0; s < 16; ++s) {
            float h = fraction * delta + left_elevation;
            float sun_top = elevation[i] + hc[s];
            if (h < sun_top) {
                float angle_delta = sun_top - h;
                float column_height = hc[s] + hc[s];
                if (angle_delta > column_height) angle_delta = column_height;
                photons = photons + angle_delta;
            }
            fraction = fraction + 0.135f;
            if (fraction >= 1.0f) {
                left = right;
                right += 1;
                if (right >= AZ) right = 0;
                left_elevation = right_elevation;
                right_elevation = horizon[right];
                delta = right_elevation - left_elevation;
                fraction = fraction - 1.0f;
            }
        }
        out[i] = photons / pm;
    }
    return 0;
}

/* The 16 float32 half-disk heights and the photon normaliser. */
int ora_half_circle(float *out16, float *photons_max)
{
    half_circle(out16);
    *photons_max = max_photons(out16);
    return 0;
}

/* FP64 frame (psr.py:29-46): rotation columns east/north/up, translation. */
static void frame64(const double *gt, const double *proj, const float *dem, int width,
                    int row, int column, double rot[3][3], double trans[3])
{
    double crs_x = gt[0] + gt[1] * column + gt[2] * row;
    double crs_y = gt[3] + gt[4] * column + gt[5] * row;
    double xp = crs_x - proj[4], yp = crs_y - proj[5];
    double rho = hypot(xp, yp);
    double latitude, longitude;
    if (rho < 1e-9) {
        latitude = proj[1];
        longitude = proj[2];
    } else {
        double c = 2.0 * atan2(rho, 2.0 * proj[3] * proj[0]);
        double sin_c = sin(c), cos_c = cos(c);
        double sin_o = sin(proj[1]), cos_o = cos(proj[1]);
        latitude = asin(cos_c * sin_o + yp * sin_c * cos_o / rho);
        longitude = proj[2] + atan2(xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c);
    }
    double cos_lat = cos(latitude), sin_lat = sin(latitude);
    double cos_lon = cos(longitude), sin_lon = sin(longitude);
    double up[3] = {cos_lat * cos_lon, cos_lat * sin_lon, sin_lat};
    double east[3] = {-sin_lon, cos_lon, 0.0};
    double north[3] = {-sin_lat * cos_lon, -sin_lat * sin_lon, cos_lat};
    double radius = proj[0] + (double)dem[(size_t)row * width + column];
    for (int k = 0; k < 3; ++k) {
        rot[k][0] = east[k];
        rot[k][1] = north[k];
        rot[k][2] = up[k];
    }
    for (int j = 0; j < 3; ++j)
        trans[j] = -(radius * up[0] * rot[0][j] + radius * up[1] * rot[1][j] +
                     radius * up[2] * rot[2][j]);
}

/* FP64 azimuth [0, 360) and elevation (deg) of vectors in a pixel frame
 * (psr.py:49-58). */
static void az_el(const double rot[3][3], const double trans[3], const double *v,
                  double *azimuth, double *elevation)
{
    double e[3];
    for (int j = 0; j < 3; ++j)
        e[j] = v[0] * rot[0][j] + v[1] * rot[1][j] + v[2] * rot[2][j] + trans[j];
    double a = atan2(e[0], e[1]) * (180.0 / M_PI);
    a = fmod(a, 360.0);
    if (a < 0.0) a += 360.0;
    *azimuth = a;
    *elevation = atan2(e[2], hypot(e[0], e[1])) * (180.0 / M_PI);
}

/* compute_psr_patch_reference (psr.py:94-140): 255 unless some vector's
 * centre elevation minus the interpolated horizon exceeds -0.545/2 deg.
 * dem float32[height, width] (whole DEM), horizons float32[vh, vw, 1440] or
 * [128,128,1440] with `stride_width` pixels per horizon row. */
int ora_psr_tile(const float *dem, int width, int height, const double *gt,
                 const double *proj, const double *vectors, int count, const float *horizons,
                 int stride_width, int tile_x, int tile_y, int valid_width, int valid_height,
                 double limb_threshold, uint8_t *out, int threads)
{
    (void)height;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
    for (int index = 0; index < valid_width * valid_height; ++index) {
        int lx = index % valid_width, ly = index / valid_width;
        double rot[3][3], trans[3];
        frame64(gt, proj, dem, width, tile_y + ly, tile_x + lx, rot, trans);
        const float *h = horizons + ((size_t)ly * stride_width + lx) * AZ;
        uint8_t value = 255;
        for (int t = 0; t < count; ++t) {
            double az, el;
            az_el(rot, trans, vectors + 3 * (size_t)t, &az, &el);
            double position = az * (AZ / 360.0);
            double fl = floor(position);
            long lower = ((long)fl % AZ + AZ) % AZ;
            long upper = (lower + 1) % AZ;
            double fraction = position - fl;
            /* The horizon difference is a float32 subtraction (NumPy keeps
             * float32 - float32 in float32); the lerp is FP64. */
            float span = h[upper] - h[lower];
            double interpolated = (double)h[lower] + fraction * (double)span;
            if (el - interpolated > limb_threshold) {
                value = 0;
                break;
            }
        }
        out[(size_t)ly * valid_width + lx] = value;
    }
    return 0;
}

/* Per pixel, the largest (centre elevation - interpolated horizon) over all
 * vectors (FP64, same arithmetic as ora_psr_tile): a pixel is PSR iff this
 * peak is <= the limb threshold; used to bound the near-threshold band. */
int ora_psr_peak(const float *dem, int width, int height, const double *gt,
                 const double *proj, const double *vectors, int count, const float *horizons,
                 int stride_width, int tile_x, int tile_y, int valid_width, int valid_height,
                 double *out, int threads)
{
    (void)height;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
    for (int index = 0; index < valid_width * valid_height; ++index) {
        int lx = index % valid_width, ly = index / valid_width;
        double rot[3][3], trans[3];
        frame64(gt, proj, dem, width, tile_y + ly, tile_x + lx, rot, trans);
        const float *h = horizons + ((size_t)ly * stride_width + lx) * AZ;
        double peak = -INFINITY;
        for (int t = 0; t < count; ++t) {
            double az, el;
            az_el(rot, trans, vectors + 3 * (size_t)t, &az, &el);
            double position = az * (AZ / 360.0);
            double fl = floor(position);
            long lower = ((long)fl % AZ + AZ) % AZ;
            long upper = (lower + 1) % AZ;
            float span = h[upper] - h[lower];
            double interpolated = (double)h[lower] + (position - fl) * (double)span;
            if (el - interpolated > peak) peak = el - interpolated;
        }
        out[(size_t)ly * valid_width + lx] = peak;
    }
    return 0;
}

/* Five viewpoints' azimuth/elevation of every vector (psr.py:61-79). */
int ora_psr_viewpoints(const float *dem, int width, int height, const double *gt,
                       const double *proj, const double *vectors, int count,
                       double *azimuth_out, double *elevation_out)
{
    int points[5][2] = {{0, 0}, {0, width - 1}, {height - 1, 0}, {height - 1, width - 1},
                        {height / 2, width / 2}};
    for (int p = 0; p < 5; ++p) {
        double rot[3][3], trans[3];
        frame64(gt, proj, dem, width, points[p][0], points[p][1], rot, trans);
        for (int t = 0; t < count; ++t)
            az_el(rot, trans, vectors + 3 * (size_t)t, azimuth_out + (size_t)p * count + t,
                  elevation_out + (size_t)p * count + t);
    }
    return 0;
}
