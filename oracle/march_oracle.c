/*
 * ORACLE — test infrastructure only.  CPU restatement of lunarscout's
 * production horizon march (one DEM pass of subpatch_hierarchy_kernel) and of
 * its factor-four max pyramid.  Only tests, the smoke check and the CPU-baseline
 * leg of the benchmark load this library; the product never does.
 *
 * Reference algorithm: src/lunarscout/_numba_horizon/cuda_backend.py:43-132,
 * :656-874, :965-1134 and src/lunarscout/_numba_horizon/pyramid.py:19-138.
 *
 * Pinned against the reference's own golden captures
 * (tests/data/numba_horizon/phase4d_production_segments.json per-DEM slopes of
 * the C# production kernel, 2 passes x 1440 azimuths, and its traversal
 * trace; phase1_reference_rays.npz pyramids), see tests/test_oracle_pins.py.
 *
 * FP32 arithmetic is written out operation by operation; the build uses
 * -ffp-contract=off so that the only fused multiply-adds are the ones this
 * file asks for through CONTRACT/LERP_FMA.  Which multiply-adds the
 * reference's GPU compiler fused is selected by a bit mask (ORA_CF_*); the
 * mask that reproduces the golden captures is the production one.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum {
    ORA_CF_EVAL = 1u << 0,   /* quartic position evaluation */
    ORA_CF_TAN = 1u << 1,    /* quartic tangent evaluation */
    ORA_CF_PLANAR = 1u << 2, /* planar distance radicand */
    ORA_CF_CHORD = 1u << 3,  /* planar->chord cubic */
    ORA_CF_TRUEM = 1u << 4,  /* chord start + cubic */
    ORA_CF_NEAR = 1u << 5,   /* true_m - block_m */
    ORA_CF_BOUND = 1u << 6,  /* 4-cell bound local-z */
    ORA_CF_SLOPE = 1u << 7,  /* level-0 sample local-z */
    ORA_CF_MAG = 1u << 8,    /* tangent magnitude radicand */
    ORA_CF_BILIN = 1u << 9,  /* bilinear lerps */
    ORA_CF_RES = 1u << 10,   /* pixel-size radicands */
    /* For a*b + c*d, the _ALT bit fuses the other product. */
    ORA_CF_PLANAR_ALT = 1u << 11,
    ORA_CF_CHORD_ALT = 1u << 12,
    ORA_CF_MAG_ALT = 1u << 13,
    ORA_CF_SLOPE_ALT = 1u << 14,
    ORA_CF_BOUND_ALT = 1u << 15,
    ORA_CF_RES_ALT = 1u << 17,
    ORA_CF_LXS_ALT = 1u << 18, /* local_x^2: fuse dist*dist instead of z*z */
    ORA_CF_SHIFT = 1u << 19,   /* subpatch shift product into the shift add */
    ORA_OPT_EXIT_CAP = 1u << 16, /* superseded level-0 cell-exit step cap */
    /* Skip ladder (this project's batched traversal, not the reference's):
     * after a cull at level l, climb to the parent levels while their
     * four-cell bound is culled too, and skip to the exit of the largest
     * culled cell.  Bits 24..27 cap the climb (0 = up to the top level). */
    ORA_OPT_LADDER = 1u << 20,
    /* Relative-height level-0 slopes (this project's accuracy mode, not the
     * reference's): the sample's local z is formed from height - observer_z
     * and 2R + height + observer_z, as the four-cell bound's is, instead of
     * from the rounded radii R + height and R + observer_z. */
    ORA_OPT_RELATIVE = 1u << 21,
};
#define ORA_LADDER_CAP(mask) (((mask) >> 24) & 15u)
/* Bits 28..31: the ladder acts only from this distance on, in km. */
#define ORA_LADDER_MIN_M(mask) (1000.0 * (double)(((mask) >> 28) & 15u))

typedef struct {
    const float *level0;
    int width, height;
    const float *mips;
    const int32_t *levels; /* [level_count, 4] = (level, offset, width, height) */
    int level_count;
    const float *map;        /* 11 map parameters */
    const float *projection; /* 6 projection parameters */
} ora_pyramid;

typedef struct {
    float *rows; /* [capacity, 12]: s, true_m, level, cx, cy, px, py, bound,
                    sample height, sample slope, advance, action */
    int capacity;
    int count;
} ora_trace;

#define ORA_TRACE(t, s_, tm_, lv_, cx_, cy_, px_, py_, mh_, h_, sl_, adv_, act_)       \
    do {                                                                               \
        if ((t) && (t)->count < (t)->capacity) {                                       \
            float *r_ = (t)->rows + (size_t)(t)->count * 12;                           \
            r_[0] = (float)(s_); r_[1] = (float)(tm_); r_[2] = (float)(lv_);           \
            r_[3] = (float)(cx_); r_[4] = (float)(cy_); r_[5] = (float)(px_);          \
            r_[6] = (float)(py_); r_[7] = (float)(mh_); r_[8] = (float)(h_);           \
            r_[9] = (float)(sl_); r_[10] = (float)(adv_); r_[11] = (float)(act_);      \
            (t)->count++;                                                              \
        }                                                                              \
    } while (0)

/* ---- FP32 instantiation: the production arithmetic ---- */
#define REAL float
#define FN(n) n##_f32
#define KC(x) ((float)(x##f))
#define SQRT sqrtf
#define FABS fabsf
#define CONTRACT(flag, a, b, c) ((mask & (flag)) ? fmaf((a), (b), (c)) : (float)((float)((a) * (b)) + (c)))
#define LERP_FMA(a, b, c) fmaf((a), (b), (c))
#include "march_body.inc"
#undef REAL
#undef FN
#undef KC
#undef SQRT
#undef FABS
#undef CONTRACT
#undef LERP_FMA

/* ---- FP64 instantiation: the same march without FP32 rounding ---- */
#define REAL double
#define FN(n) n##_f64
#define KC(x) ((double)(x))
#define SQRT sqrt
#define FABS fabs
#define CONTRACT(flag, a, b, c) ((void)mask, (a) * (b) + (c))
#define LERP_FMA(a, b, c) ((a) * (b) + (c))
#include "march_body.inc"
#undef REAL
#undef FN
#undef KC
#undef SQRT
#undef FABS
#undef CONTRACT
#undef LERP_FMA

static void make_pyramid(ora_pyramid *p, const float *level0, int width, int height,
                         const float *mips, const int32_t *levels, int level_count,
                         const float *map, const float *projection)
{
    p->level0 = level0;
    p->width = width;
    p->height = height;
    p->mips = mips;
    p->levels = levels;
    p->level_count = level_count;
    p->map = map;
    p->projection = projection;
}

/*
 * One DEM pass over a tile (all pixels x all azimuths when `pixels` is NULL,
 * else the listed (pixel, azimuth) pairs).  `slopes` carries the previous
 * pass's values in and this pass's out: [tile_width*tile_height, A] for the
 * full tile or [n] for a list.  Returns 0.
 */
#define ORA_MARCH_ARGS                                                                  \
    const float *segments, int azimuth_count, int center_count, int dem_count,           \
        const float *p_level0, int p_width, int p_height, const float *p_map,            \
        const float *a_level0, int a_width, int a_height, const float *a_mips,           \
        const int32_t *a_levels, int a_level_count, const float *a_map,                  \
        const float *a_projection, int tile_column, int tile_row, int tile_width,        \
        int tile_height, int subpatch, int pass_index, float observer_elevation,         \
        const int32_t *pixels, const int32_t *azimuths, long long n

#define ORA_MARCH_BODY(SUFFIX, TYPE)                                                     \
    ora_pyramid primary, active;                                                         \
    make_pyramid(&primary, p_level0, p_width, p_height, NULL, NULL, 0, p_map, NULL);     \
    make_pyramid(&active, a_level0, a_width, a_height, a_mips, a_levels, a_level_count,  \
                 a_map, a_projection);                                                   \
    const long long pixel_count = (long long)tile_width * tile_height;                   \
    const long long total = pixels ? n : pixel_count * azimuth_count;                    \
    long long visits = 0, samples = 0;                                                   \
    _Pragma("omp parallel for schedule(dynamic, 64) num_threads(threads) reduction(+:visits, samples)") \
    for (long long i = 0; i < total; ++i) {                                              \
        int pixel, azimuth;                                                              \
        long long out;                                                                   \
        if (pixels) {                                                                    \
            pixel = pixels[i];                                                           \
            azimuth = azimuths[i];                                                       \
            out = i;                                                                     \
        } else {                                                                         \
            pixel = (int)(i % pixel_count);                                              \
            azimuth = (int)(i / pixel_count);                                            \
            out = (long long)pixel * azimuth_count + azimuth;                            \
        }                                                                                \
        TYPE value = slopes[out];                                                        \
        long long c[2] = {0, 0};                                                         \
        if (march_one_##SUFFIX(segments, azimuth_count, center_count, dem_count,         \
                               &primary, &active, tile_column, tile_row, tile_width,    \
                               subpatch, pass_index, observer_elevation, pixel,         \
                               azimuth, &value, mask, c, NULL))                          \
            slopes[out] = value;                                                         \
        visits += c[0];                                                                  \
        samples += c[1];                                                                 \
    }                                                                                    \
    if (counters) {                                                                      \
        counters[0] = visits;                                                            \
        counters[1] = samples;                                                           \
    }                                                                                    \
    return 0;

int ora_march_pass_f32(ORA_MARCH_ARGS, float *slopes, unsigned mask, int threads,
                       long long *counters)
{
    if (threads < 1) threads = 1;
    ORA_MARCH_BODY(f32, float)
}

int ora_march_pass_f64(ORA_MARCH_ARGS, double *slopes, unsigned mask, int threads,
                       long long *counters)
{
    if (threads < 1) threads = 1;
    ORA_MARCH_BODY(f64, double)
}

/* One ray with its branch trace (action codes of the reference's
 * hierarchy trace: 0 descend, 1 culled, 2 no data, 3 out of bounds,
 * 4 level-0 sample).  Returns the trace length. */
int ora_march_trace_f32(ORA_MARCH_ARGS, float *slope_inout, unsigned mask,
                        float *trace_rows, int capacity)
{
    (void)n;
    ora_pyramid primary, active;
    make_pyramid(&primary, p_level0, p_width, p_height, NULL, NULL, 0, p_map, NULL);
    make_pyramid(&active, a_level0, a_width, a_height, a_mips, a_levels, a_level_count,
                 a_map, a_projection);
    ora_trace trace = {trace_rows, capacity, 0};
    (void)tile_height;
    march_one_f32(segments, azimuth_count, center_count, dem_count, &primary, &active,
                  tile_column, tile_row, tile_width, subpatch, pass_index,
                  observer_elevation, pixels[0], azimuths[0], slope_inout, mask, NULL,
                  &trace);
    return trace.count;
}

/* The same in FP64 (the trace rows are stored as float32). */
int ora_march_trace_f64(ORA_MARCH_ARGS, double *slope_inout, unsigned mask,
                        float *trace_rows, int capacity)
{
    (void)n;
    ora_pyramid primary, active;
    make_pyramid(&primary, p_level0, p_width, p_height, NULL, NULL, 0, p_map, NULL);
    make_pyramid(&active, a_level0, a_width, a_height, a_mips, a_levels, a_level_count,
                 a_map, a_projection);
    ora_trace trace = {trace_rows, capacity, 0};
    (void)tile_height;
    march_one_f64(segments, azimuth_count, center_count, dem_count, &primary, &active,
                  tile_column, tile_row, tile_width, subpatch, pass_index,
                  observer_elevation, pixels[0], azimuths[0], slope_inout, mask, NULL,
                  &trace);
    return trace.count;
}

/* The bare march of one already-interpolated 16-field segment
 * (start_x, start_y, a1..a4, b1..b4, s_start, s_end, s_start_chord, c1..c3). */
float ora_hierarchy_maximum_f32(const float *segment16, const float *level0, int width,
                                int height, const float *mips, const int32_t *levels,
                                int level_count, float observer_z, float radius,
                                float resolution, int pass_index, float initial,
                                unsigned mask, float *trace_rows, int capacity,
                                int *trace_count)
{
    ora_pyramid p;
    make_pyramid(&p, level0, width, height, mips, levels, level_count, NULL, NULL);
    ora_trace trace = {trace_rows, capacity, 0};
    float seg[16];
    memcpy(seg, segment16, sizeof seg);
    float r = hierarchy_maximum_f32(seg, &p, observer_z, radius, resolution, pass_index,
                                    initial, mask, NULL, trace_rows ? &trace : NULL, 0, 0);
    if (trace_count) *trace_count = trace.count;
    return r;
}

/* ---- factor-four max pyramid (pyramid.py:19-31,110-138) ---- */

/* Level table: (level, offset into mips, width, height).  Returns the level
 * count; *mip_count receives the total mip elements.  `levels` may be NULL to
 * query the count. */
int ora_pyramid_layout(int width, int height, int32_t *levels, long long *mip_count)
{
    int count = 0;
    long long offset = 0;
    int w = width, h = height;
    for (;;) {
        if (levels) {
            levels[count * 4 + 0] = count;
            levels[count * 4 + 1] = count == 0 ? 0 : (int32_t)offset;
            levels[count * 4 + 2] = w;
            levels[count * 4 + 3] = h;
        }
        if (count > 0) offset += (long long)w * h;
        ++count;
        if (w == 1 && h == 1) break;
        w = (w + 3) / 4;
        h = (h + 3) / 4;
    }
    if (mip_count) *mip_count = offset;
    return count;
}

static int pyr_valid(float v) { return !isnan(v) && !isinf(v) && v > -20000.0f; }

/* Each level-l cell is the max of the valid cells of its 4x4 block of level
 * l-1; a block without a valid cell is -32000. */
int ora_build_pyramid(const float *level0, int width, int height, float *mips)
{
    int32_t levels[4 * 40];
    long long mip_count = 0;
    int count = ora_pyramid_layout(width, height, levels, &mip_count);
    const float *src = level0;
    int sw = width, sh = height;
    for (int l = 1; l < count; ++l) {
        int dw = levels[l * 4 + 2], dh = levels[l * 4 + 3];
        float *dst = mips + levels[l * 4 + 1];
        for (int y = 0; y < dh; ++y) {
            for (int x = 0; x < dw; ++x) {
                float best = -32000.0f;
                for (int dy = 0; dy < 4; ++dy) {
                    int yy = y * 4 + dy;
                    if (yy >= sh) break;
                    for (int dx = 0; dx < 4; ++dx) {
                        int xx = x * 4 + dx;
                        if (xx >= sw) break;
                        float v = src[(size_t)yy * sw + xx];
                        if (pyr_valid(v) && v > best) best = v;
                    }
                }
                dst[(size_t)y * dw + x] = best;
            }
        }
        src = dst;
        sw = dw;
        sh = dh;
    }
    return count;
}
