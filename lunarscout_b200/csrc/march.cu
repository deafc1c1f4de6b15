// Production horizon march for sm_100a: one DEM pass of the hierarchical,
// adaptive ray march over a 128x128 tile x 1440 azimuths.
//
// Semantics follow src/lunarscout/_numba_horizon/cuda_backend.py:
//   subpatch_hierarchy_kernel :1007-1134 (segment interpolation, observer)
//   hierarchy_maximum          :656-874  (the march)
//   helpers                    :43-132
//
// Arithmetic contract.  This file is compiled with --fmad=false, so every
// written multiply and add rounds separately, and the multiply-adds that the
// reference's GPU compiler fuses are written as explicit __fmaf_rn:
//   * every "x + a*b" / "x - a*b" whose product feeds the add is fused;
//   * for "a*b + c*d" the first product is fused.
// Division, reciprocal and square root are IEEE round-to-nearest.  With the
// same segment inputs the results are bit-identical to the CPU oracle's FP32
// restatement, which reproduces the reference's golden traversal captures.
//
// The kernel is bound by instruction issue (its gathers hit L1/L2), so the
// work per node visit is kept small without changing any rounded value or
// decision:
//   * cells come from a sanitized copy of level 0 (invalid -> -32000) packed
//     with the mips, so validity is one comparison and the four-cell bound
//     is a plain maximum;
//   * per-level constants (cell side, block metres, step and fallback
//     advances, offsets) live in a shared table computed once per block;
//   * the tangent and its reciprocals depend only on the ray position and are
//     computed once per position, not per level;
//   * the cull test decides with a cheap bound outside a guard band and with
//     the reference arithmetic inside it (bound_culled).
//
// Layout.  Working slopes are azimuth-major [A, P] so that a warp (32
// adjacent pixels of one tile row, one azimuth) reads and writes 128
// contiguous bytes; a transpose kernel produces the reference's pixel-major
// [P, A] at the end.  The first pass writes without reading (the reference
// resets the buffer to -inf before pass 0).
#include "internal.cuh"

namespace ls200 {

struct MarchParams {
    const float *segments;  // [A, C, D, 18]
    int azimuth_count, center_count, dem_count;
    const float *primary_cells;
    int primary_width, primary_height;
    float primary_m6, primary_m9;
    const float *cells;  // sanitized level 0 + mips of the active DEM
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

// Per-level constants shared by a block (every thread of a launch marches
// the same DEM at the same resolution).
struct LevelTable {
    float side[kMaxLevels];      // float(4^l) * resolution: the level choice
    float block_m[kMaxLevels];   // the same product (metres per cell)
    float fallback[kMaxLevels];  // ((block_m * 0.5) * 0.001)
    float out_step[kMaxLevels];  // max(0.001, block_m * 0.001)
    int4 cells[kMaxLevels];      // (offset, width, height, -)
};

__device__ __forceinline__ float quartic(float x0, float a1, float a2, float a3, float a4,
                                         float d) {
    const float d2 = __fmul_rn(d, d);
    const float d3 = __fmul_rn(d2, d);
    const float d4 = __fmul_rn(d2, d2);
    float r = __fmaf_rn(a1, d, x0);
    r = __fmaf_rn(a2, d2, r);
    r = __fmaf_rn(a3, d3, r);
    return __fmaf_rn(a4, d4, r);
}

__device__ __forceinline__ float quartic_tangent(float a1, float a2, float a3, float a4,
                                                 float d) {
    const float d2 = __fmul_rn(d, d);
    const float d3 = __fmul_rn(d2, d);
    float r = __fmaf_rn(__fmul_rn(2.0f, a2), d, a1);
    r = __fmaf_rn(__fmul_rn(3.0f, a3), d2, r);
    return __fmaf_rn(__fmul_rn(4.0f, a4), d3, r);
}

// Clamped bilinear sample of sanitized level-0 cells; -32000 when any corner
// is invalid (cuda_backend.py:107-132).
__device__ __forceinline__ float bilinear(const float *__restrict__ cells, int width,
                                          int height, float column, float row) {
    const float cmax = __fsub_rn(static_cast<float>(width), 1.0001f);
    const float rmax = __fsub_rn(static_cast<float>(height), 1.0001f);
    column = column > 0.0f ? column : 0.0f;
    column = column < cmax ? column : cmax;
    row = row > 0.0f ? row : 0.0f;
    row = row < rmax ? row : rmax;
    const int x0 = static_cast<int>(floorf(column));
    const int y0 = static_cast<int>(floorf(row));
    const int x1 = min(x0 + 1, width - 1);
    const int y1 = min(y0 + 1, height - 1);
    const float *r0 = cells + static_cast<size_t>(y0) * width;
    const float *r1 = cells + static_cast<size_t>(y1) * width;
    const float q00 = __ldg(r0 + x0), q10 = __ldg(r0 + x1);
    const float q01 = __ldg(r1 + x0), q11 = __ldg(r1 + x1);
    if (!(q00 > -20000.0f && q10 > -20000.0f && q01 > -20000.0f && q11 > -20000.0f))
        return -32000.0f;
    const float tx = __fsub_rn(column, static_cast<float>(x0));
    const float ty = __fsub_rn(row, static_cast<float>(y0));
    const float top = __fmaf_rn(tx, __fsub_rn(q10, q00), q00);
    const float bottom = __fmaf_rn(tx, __fsub_rn(q11, q01), q01);
    return __fmaf_rn(ty, __fsub_rn(bottom, top), top);
}

// Local-z slope of a terrain point seen over the chord `dist`
// (cuda_backend.py:812-830): numerator fused on its first product, local_x^2
// fused on dist*dist.
__device__ __forceinline__ float sample_slope(float dist, float height, float radius,
                                              float observer_radius) {
    const float squared = __fmul_rn(dist, dist);
    const float point_radius = __fadd_rn(radius, height);
    const float radius_delta = __fsub_rn(point_radius, observer_radius);
    const float radius_sum = __fadd_rn(point_radius, observer_radius);
    const float numerator = __fmaf_rn(radius_delta, radius_sum, -squared);
    const float local_z = __fdiv_rn(numerator, __fmul_rn(2.0f, observer_radius));
    const float lx2 = __fmaf_rn(dist, dist, -__fmul_rn(local_z, local_z));
    const float local_x = lx2 > 0.0f ? __fsqrt_rn(lx2) : 1e-6f;
    return __fdiv_rn(local_z, local_x);
}

// The same for the four-cell culling bound (cuda_backend.py:777-795).
__device__ __forceinline__ float bound_slope(float dist, float height, float radius,
                                             float observer_z, float observer_radius) {
    const float squared = __fmul_rn(dist, dist);
    const float height_delta = __fsub_rn(height, observer_z);
    float radius_sum = __fadd_rn(__fmul_rn(2.0f, radius), height);
    radius_sum = __fadd_rn(radius_sum, observer_z);
    const float numerator = __fmaf_rn(height_delta, radius_sum, -squared);
    const float local_z = __fdiv_rn(numerator, __fmul_rn(2.0f, observer_radius));
    const float lx2 = __fmaf_rn(dist, dist, -__fmul_rn(local_z, local_z));
    const float local_x = lx2 > 0.0f ? __fsqrt_rn(lx2) : 1e-6f;
    return __fdiv_rn(local_z, local_x);
}

// Exactly `possible <= current` for the four-cell bound `possible` of the
// reference (near field: fl((h - oz) / tn); far field: bound_slope), at a
// fraction of its cost.  The cull test is the most frequent operation of the
// march and `possible` only feeds this comparison, so an approximation may
// decide it whenever it lies outside a guard band around `current`:
//   near: __fdividef has at most 2 ulp error;
//   far:  the numerator is the exact one; z = num * rcp(den) is within 3 ulp
//         of fl(num / den); with local_x^2 > tn^2 / 4 (bound below 60 deg)
//         the cancellation in local_x^2 amplifies that by at most 3, and
//         rsqrtf adds 2 ulp: the approximation is within 2e-6 (relative) of
//         the exact FP32 value.
// The band is 1e-5 relative, five times that bound; inside it, and for
// steeper bounds, the exact arithmetic of the reference decides.
__device__ __forceinline__ bool bound_culled(bool near, float true_near, float height,
                                             float radius, float observer_z,
                                             float observer_radius, float inverse_denominator,
                                             float current) {
    float approx;
    if (near) {
        approx = __fdividef(__fsub_rn(height, observer_z), true_near);
    } else {
        const float squared = __fmul_rn(true_near, true_near);
        const float height_delta = __fsub_rn(height, observer_z);
        float radius_sum = __fadd_rn(__fmul_rn(2.0f, radius), height);
        radius_sum = __fadd_rn(radius_sum, observer_z);
        const float numerator = __fmaf_rn(height_delta, radius_sum, -squared);
        const float local_z = __fmul_rn(numerator, inverse_denominator);
        const float lx2 = __fmaf_rn(true_near, true_near, -__fmul_rn(local_z, local_z));
        if (!(lx2 > 0.25f * squared)) {
            return bound_slope(true_near, height, radius, observer_z, observer_radius) <= current;
        }
        approx = __fmul_rn(local_z, rsqrtf(lx2));
    }
    const float band = 1e-5f * fmaxf(fabsf(approx), fabsf(current));
    if (approx < current - band) return true;
    if (approx > current + band) return false;
    const float possible =
        near ? __fdiv_rn(__fsub_rn(height, observer_z), true_near)
             : bound_slope(true_near, height, radius, observer_z, observer_radius);
    return possible <= current;
}

__device__ __forceinline__ int clamp_center(int requested, int dem_size, int subpatch) {
    const int half = subpatch / 2;
    int maximum = dem_size - half;
    if (maximum < half) maximum = half;
    if (requested < half) return half;
    if (requested > maximum) return maximum;
    return requested;
}

__device__ __forceinline__ float hypot_fused(float a, float b) {
    return __fsqrt_rn(__fmaf_rn(a, a, __fmul_rn(b, b)));
}

template <bool kCount>
__global__ void __launch_bounds__(128, 8) march_pass_kernel(const __grid_constant__ MarchParams P) {
    __shared__ LevelTable table;
    const float column_res = hypot_fused(P.m6, P.m9);
    const float row_res = hypot_fused(P.m7, P.m10);
    const float resolution = __fmul_rn(__fadd_rn(column_res, row_res), 0.5f);
    if (threadIdx.x < P.level_count) {
        const int l = threadIdx.x;
        const float block_m = __fmul_rn(static_cast<float>(1 << (2 * l)), resolution);
        const float step_km = __fmul_rn(block_m, 0.001f);
        table.side[l] = block_m;
        table.block_m[l] = block_m;
        table.fallback[l] = __fmul_rn(__fmul_rn(block_m, 0.5f), 0.001f);
        table.out_step[l] = 0.001f > step_km ? 0.001f : step_km;
        table.cells[l] = P.levels[l];
    }
    __syncthreads();

    const int pixel_count = P.tile_width * P.tile_height;
    const long long linear = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (linear >= static_cast<long long>(pixel_count) * P.azimuth_count) return;
    const int pixel = static_cast<int>(linear % pixel_count);
    const int azimuth = static_cast<int>(linear / pixel_count);
    const int row = pixel / P.tile_width;
    const int column = pixel % P.tile_width;
    float *out = P.slopes + static_cast<size_t>(azimuth) * pixel_count + pixel;
    // Pixels outside the primary DEM keep the initial -inf sentinel.
    if (P.tile_column + column >= P.primary_width || P.tile_row + row >= P.primary_height) {
        if (P.first_pass) *out = -INFINITY;
        return;
    }

    // ---- subpatch interpolation (cuda_backend.py:1032-1119) ----
    const int count = P.tile_width / P.subpatch + 2;
    const float gx = __fadd_rn(__fdiv_rn(static_cast<float>(column - P.subpatch / 2),
                                         static_cast<float>(P.subpatch)), 1.0f);
    const float gy = __fadd_rn(__fdiv_rn(static_cast<float>(row - P.subpatch / 2),
                                         static_cast<float>(P.subpatch)), 1.0f);
    int left = static_cast<int>(gx), top = static_cast<int>(gy);
    float tx = __fsub_rn(gx, static_cast<float>(left));
    float ty = __fsub_rn(gy, static_cast<float>(top));
    if (left < 0) { left = 0; tx = 0.0f; }
    if (top < 0) { top = 0; ty = 0.0f; }
    if (left > count - 2) { left = count - 2; tx = 1.0f; }
    if (top > count - 2) { top = count - 2; ty = 1.0f; }
    const int i00 = top * count + left, i10 = i00 + 1;
    const int i01 = (top + 1) * count + left, i11 = i01 + 1;
    const float ratio = __fdiv_rn(hypot_fused(P.primary_m6, P.primary_m9), column_res);
    const int req_left = P.tile_column + (left - 1) * P.subpatch + P.subpatch / 2;
    const int req_top = P.tile_row + (top - 1) * P.subpatch + P.subpatch / 2;
    const float d_left = static_cast<float>(
        column - (clamp_center(req_left, P.primary_width, P.subpatch) - P.tile_column));
    const float d_right = static_cast<float>(
        column - (clamp_center(req_left + P.subpatch, P.primary_width, P.subpatch) -
                  P.tile_column));
    const float d_top = static_cast<float>(
        row - (clamp_center(req_top, P.primary_height, P.subpatch) - P.tile_row));
    const float d_bottom = static_cast<float>(
        row - (clamp_center(req_top + P.subpatch, P.primary_height, P.subpatch) -
               P.tile_row));

    const size_t stride_c = static_cast<size_t>(P.dem_count) * kSegmentFields;
    const float *base = P.segments +
                        static_cast<size_t>(azimuth) * P.center_count * stride_c +
                        static_cast<size_t>(P.pass_index) * kSegmentFields;
    const float *s00 = base + i00 * stride_c, *s10 = base + i10 * stride_c;
    const float *s01 = base + i01 * stride_c, *s11 = base + i11 * stride_c;
    float seg[kMarchFields];
#pragma unroll
    for (int k = 0; k < kMarchFields; ++k) {
        const int f = k < 2 ? k : k + 2;
        float v00 = __ldg(s00 + f), v10 = __ldg(s10 + f);
        float v01 = __ldg(s01 + f), v11 = __ldg(s11 + f);
        if (f == 0) {
            v00 = __fmaf_rn(d_left, ratio, v00);
            v10 = __fmaf_rn(d_right, ratio, v10);
            v01 = __fmaf_rn(d_left, ratio, v01);
            v11 = __fmaf_rn(d_right, ratio, v11);
        } else if (f == 1) {
            v00 = __fmaf_rn(d_top, ratio, v00);
            v10 = __fmaf_rn(d_top, ratio, v10);
            v01 = __fmaf_rn(d_bottom, ratio, v01);
            v11 = __fmaf_rn(d_bottom, ratio, v11);
        }
        const float upper = __fmaf_rn(__fsub_rn(v10, v00), tx, v00);
        const float lower = __fmaf_rn(__fsub_rn(v11, v01), tx, v01);
        seg[k] = __fmaf_rn(__fsub_rn(lower, upper), ty, upper);
    }
    const float start_x = seg[0], start_y = seg[1];
    const float a1 = seg[2], a2 = seg[3], a3 = seg[4], a4 = seg[5];
    const float b1 = seg[6], b2 = seg[7], b3 = seg[8], b4 = seg[9];
    const float s_start = seg[10], s_end = seg[11], s_start_chord = seg[12];
    const float c1 = seg[13], c2 = seg[14], c3 = seg[15];

    const float observer_z = __fadd_rn(
        bilinear(P.primary_cells, P.primary_width, P.primary_height,
                 static_cast<float>(P.tile_column + column),
                 static_cast<float>(P.tile_row + row)),
        P.observer_elevation);
    const float radius = P.radius;
    const float observer_radius = __fadd_rn(radius, observer_z);
    const float inverse_denominator = __frcp_rn(__fmul_rn(2.0f, observer_radius));
    const float *__restrict__ cells = P.cells;

    // ---- hierarchy_maximum (cuda_backend.py:656-874) ----
    float current = -1e30f;
    if (!P.first_pass) {
        const float initial = *out;
        current = isinf(initial) ? -1e30f : initial;
    }
    float s = s_start > 0.001f ? s_start : 0.001f;
    const float minimum_step = __fmul_rn(__fmul_rn(0.5f, resolution), 0.001f);
    const float primary_far_step = __fmul_rn(__fmul_rn(0.8f, resolution), 0.001f);
    const float last_x = static_cast<float>(P.width - 1);
    const float last_y = static_cast<float>(P.height - 1);
    const int top_level = P.level_count - 1;
    int level_hint = top_level;
    unsigned visits = 0, samples = 0, steps = 0;
    while (s <= s_end) {
        if (kCount) ++steps;
        const float delta = __fsub_rn(s, s_start);
        const float px = quartic(start_x, a1, a2, a3, a4, delta);
        const float py = quartic(start_y, b1, b2, b3, b4, delta);
        // NaN fails every comparison, as the reference's isnan tests do.
        if (!(px >= 0.0f && py >= 0.0f && px < last_x && py < last_y)) break;
        const float planar_x = __fmul_rn(__fsub_rn(px, start_x), resolution);
        const float planar_y = __fmul_rn(__fsub_rn(py, start_y), resolution);
        const float planar_m = hypot_fused(planar_x, planar_y);
        const bool near = s < 0.5f;
        float true_m;
        if (near) {
            true_m = __fmul_rn(s, 1000.0f);
        } else {
            const float pm2 = __fmul_rn(planar_m, planar_m);
            const float pm3 = __fmul_rn(pm2, planar_m);
            float chord = __fmaf_rn(c1, planar_m, __fmul_rn(c2, pm2));
            chord = __fmaf_rn(c3, pm3, chord);
            true_m = __fmaf_rn(s_start_chord, 1000.0f, chord);
        }
        const float footprint = __fmul_rn(true_m, 0.004363323129985824f);
        // The reference scans down from the top level to the largest level
        // whose side fits the footprint (or 0).  Sides grow with the level,
        // so that level is also found by moving up or down from the previous
        // step's level, which usually takes one comparison.
        int level = level_hint;
        while (level < top_level && table.side[level + 1] <= footprint) ++level;
        while (level > 0 && !(table.side[level] <= footprint)) --level;
        level_hint = level;
        // The tangent and its reciprocals depend only on delta.
        const float dx = quartic_tangent(a1, a2, a3, a4, delta);
        const float dy = quartic_tangent(b1, b2, b3, b4, delta);
        const float inv_x = fabsf(dx) > 1e-8f ? __frcp_rn(dx) : 1e30f;
        const float inv_y = fabsf(dy) > 1e-8f ? __frcp_rn(dy) : 1e30f;
        const int ipx = static_cast<int>(px), ipy = static_cast<int>(py);
        bool ray_out = false;
        for (;;) {
            const int4 L = table.cells[level];
            const int shift = level * 2;
            const int cx = ipx >> shift, cy = ipy >> shift;
            if (kCount) ++visits;
            if (cx >= L.y || cy >= L.z) {  // cx, cy >= 0 since px, py >= 0
                s = __fadd_rn(s, table.out_step[level]);
                ray_out = true;
                break;
            }
            // Four-cell bound of every bilinear sample cornered in this cell.
            const int index = L.x + cy * L.y + cx;
            const bool has_right = cx + 1 < L.y, has_down = cy + 1 < L.z;
            const float v00 = __ldg(cells + index);
            const float v10 = has_right ? __ldg(cells + index + 1) : -32000.0f;
            const float v01 = has_down ? __ldg(cells + index + L.y) : -32000.0f;
            const float v11 = has_right && has_down ? __ldg(cells + index + L.y + 1) : -32000.0f;
            const float maximum_height = fmaxf(fmaxf(v00, v10), fmaxf(v01, v11));
            // Slab exit (cuda_backend.py:733-751).  Of max(t1, t2) only the
            // far edge can win: (min_x - px) <= 0 < (max_x - px), so the
            // product with inv_x keeps that order's sign pattern and the
            // larger t is the edge ahead of the ray (bitwise the same value,
            // including the -0.0 of a ray starting on the edge).
            const float scale_f = static_cast<float>(1 << shift);
            const float min_x = static_cast<float>(cx << shift);
            const float min_y = static_cast<float>(cy << shift);
            const float edge_x = inv_x > 0.0f ? __fadd_rn(min_x, scale_f) : min_x;
            const float edge_y = inv_y > 0.0f ? __fadd_rn(min_y, scale_f) : min_y;
            const float tmx = __fmul_rn(__fsub_rn(edge_x, px), inv_x);
            const float tmy = __fmul_rn(__fsub_rn(edge_y, py), inv_y);
            const float exit_distance = tmx < tmy ? tmx : tmy;
            const float fallback = table.fallback[level];
            const float to_exit = exit_distance > 0.0f ? exit_distance : fallback;
            const float skip = to_exit > 0.0f ? __fadd_rn(to_exit, 0.0001f) : fallback;
            if (maximum_height < -20000.0f) {
                s = __fadd_rn(s, skip);
                break;
            }
            float true_near = __fmaf_rn(-scale_f, resolution, true_m);
            true_near = true_near > 1.0f ? true_near : 1.0f;
            if (bound_culled(near, true_near, maximum_height, radius, observer_z,
                             observer_radius, inverse_denominator, current)) {
                s = __fadd_rn(s, skip);
                break;
            }
            if (level == 0) {
                if (kCount) ++samples;
                const float height = bilinear(cells, P.width, P.height, px, py);
                float slope = -1e30f;
                if (height > -20000.0f) {
                    slope = near ? __fdiv_rn(__fsub_rn(height, observer_z), true_m)
                                 : sample_slope(true_m, height, radius, observer_radius);
                    if (slope > current) current = slope;
                }
                const float magnitude = hypot_fused(dx, dy);
                const float pixel_step = magnitude > 1e-6f ? __frcp_rn(magnitude) : 0.0005f;
                const float margin = __fsub_rn(current, slope);
                const float margin_step =
                    margin > 0.0f
                        ? __fdiv_rn(__fmul_rn(__fmul_rn(margin, true_m), 1.732f), 1000.0f)
                        : 0.0f;
                const float angular_step = __fdiv_rn(__fmul_rn(true_m, 0.00151f), 1000.0f);
                const float inner = margin_step < angular_step ? margin_step : angular_step;
                float advance = pixel_step > inner ? pixel_step : inner;
                if (near) advance = __fmul_rn(advance, 0.25f);
                const float floor_step =
                    (P.pass_index == 0 && true_m >= 100.0f) ? primary_far_step : minimum_step;
                advance = advance > floor_step ? advance : floor_step;
                s = __fadd_rn(s, advance);
                break;
            }
            --level;
        }
        if (ray_out) break;
    }
    *out = current > -1e29f ? current : -INFINITY;
    if (kCount) {
        // Warp-aggregated over the lanes that reach this point together
        // (counting launches are diagnostics, never timed).
        const unsigned mask = __activemask();
        const unsigned v = __reduce_add_sync(mask, visits);
        const unsigned n = __reduce_add_sync(mask, samples);
        const unsigned t = __reduce_add_sync(mask, steps);
        if ((threadIdx.x & 31) == __ffs(mask) - 1) {
            atomicAdd(P.counters, static_cast<unsigned long long>(v));
            atomicAdd(P.counters + 1, static_cast<unsigned long long>(n));
            atomicAdd(P.counters + 2, static_cast<unsigned long long>(t));
        }
    }
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
        static_cast<long long>(tile.tile_width) * tile.tile_height * tile.azimuth_count;
    const unsigned blocks = static_cast<unsigned>((total + 127) / 128);
    if (ctx->counting)
        march_pass_kernel<true><<<blocks, 128, 0, ctx->stream>>>(P);
    else
        march_pass_kernel<false><<<blocks, 128, 0, ctx->stream>>>(P);
    LS_CUDA(cudaGetLastError());
}

}  // namespace ls200
