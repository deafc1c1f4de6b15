// The per-ray core of the horizon march, shared by the per-tile production
// kernel (march.cu) and the persistent multi-site kernel (march_batch.cu).
//
// Semantics follow src/lunarscout/_numba_horizon/cuda_backend.py:
//   subpatch_hierarchy_kernel :1007-1134 (segment interpolation, observer)
//   hierarchy_maximum          :656-874  (the march)
//   helpers                    :43-132
//
// Arithmetic contract.  The including files are compiled with --fmad=false,
// so every written multiply and add rounds separately, and the multiply-adds
// that the reference's GPU compiler fuses are written as explicit __fmaf_rn:
//   * every "x + a*b" / "x - a*b" whose product feeds the add is fused;
//   * for "a*b + c*d" the first product is fused, except local_x^2 =
//     dist*dist - local_z^2, which fuses local_z^2.
// That is the reference's Numba-CUDA kernel as NVVM compiles it on the B200
// (its slopes on the same GPU are the golden file numba_cuda_b200.npz of the
// tests).  Division, reciprocal and square root are IEEE round-to-nearest;
// the tangent's reciprocals come from rcp.approx plus one Newton step, which
// equals the IEEE reciprocal on every input it receives (see rcp_approx).
// The x and y arithmetic of a step (path position and tangent, planar
// offset, cell-exit slab) is issued as f32x2 pairs, whose lanes round as the
// scalar intrinsics do.  No shift amount is ever taken from stored state:
// an amount out of range is undefined even on a path that is never taken.
// With the same segment inputs the results are bit-identical to the CPU
// oracle's FP32 restatement under its production mask.
//
// The march is bound by instruction issue (its gathers hit L1/L2), so the
// work per node visit is kept small without changing any rounded value or
// decision:
//   * cells come from a sanitized copy of level 0 (invalid -> -32000) packed
//     with the mips, so validity is one comparison and the four-cell bound
//     is a plain maximum;
//   * per-level constants (cell side, step and fallback advances, offsets)
//     come from a table computed once per DEM;
//   * the tangent and its reciprocals depend only on the ray position and are
//     computed once per position, not per level;
//   * the cull test decides with a cheap bound outside a guard band and with
//     the reference arithmetic inside it (bound_culled).
//
// The skip ladder (kLadder, the batched traversal; no reference counterpart)
// extends a cull to the largest culled ancestor cell, see ladder_advance.
//
// The relative arithmetic (kRelative; no reference counterpart) marches the
// same algorithm in FP32 on coordinates and heights relative to a local
// origin: positions as an integer origin (near the ray start) plus small
// offsets, level-0 heights as differences from the observer's z taken
// before interpolation, and the far-field local z from that difference
// (never rounding R + height on its own).  The FP32 reference arithmetic
// rounds absolute coordinates (an ulp of 5e-4 px at 4096 px) and absolute
// heights, which at the 1 m first sample moves the slope by up to ~0.02 deg;
// the relative march stays within ~1e-4 deg of the FP64 restatement.
#pragma once

#include "internal.cuh"

namespace ls200 {

// Per-level constants of one DEM.
struct LevelTable {
    float side[kMaxLevels];      // float(4^l) * resolution: the level choice
    float fallback[kMaxLevels];  // ((side * 0.5) * 0.001)
    float out_step[kMaxLevels];  // max(0.001, side * 0.001)
    int4 cells[kMaxLevels];      // (cell offset, width, height, fallback bits)
};

// Everything the march of one DEM pass needs about the DEM.
struct DemView {
    const float *cells;   // sanitized level 0 + packed mips
    const float *bounds;  // four-cell bound of every cell, the layout of cells
    int width, height, level_count;
    float resolution;    // mean pixel size of the DEM (m)
    float column_res;    // hypot of the column axis of the geotransform
    float radius;
};

// The ladder acts from this distance on (m); nearer, steep crater walls make
// the reference's slope formula sensitive to where samples fall.
constexpr float kLadderMinimumDistance = 1000.0f;

// Warp-aggregated counter update over the lanes that reach it together
// (counting launches are diagnostics, never timed).
__device__ __forceinline__ void add_counters(unsigned long long *counters, unsigned visits,
                                             unsigned samples, unsigned steps) {
    const unsigned mask = __activemask();
    const unsigned v = __reduce_add_sync(mask, visits);
    const unsigned n = __reduce_add_sync(mask, samples);
    const unsigned t = __reduce_add_sync(mask, steps);
    if ((threadIdx.x & 31) == __ffs(mask) - 1) {
        atomicAdd(counters, static_cast<unsigned long long>(v));
        atomicAdd(counters + 1, static_cast<unsigned long long>(n));
        atomicAdd(counters + 2, static_cast<unsigned long long>(t));
    }
}

// Correctly rounded reciprocal: the hardware approximation plus one
// Newton-Raphson correction whose residual an FMA forms exactly,
// y' = y + y (1 - x y) with y ~ 1/x (P. W. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Develop. 34(1), 1990).  For 2^-64 <= |x| < 2^64 it equals __frcp_rn bit for
// bit; |x| >= 2^64, infinities and NaN take __frcp_rn itself.
// ls200_check_arithmetic compares every pattern with |x| >= 2^-64.
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float hypot_fused(float a, float b) {
    return __fsqrt_rn(__fmaf_rn(a, a, __fmul_rn(b, b)));
}

// Mean pixel size (m) from the geotransform terms m6, m7 (column axis) and
// m9, m10 (row axis) (cuda_backend.py:1036-1040).
__device__ __forceinline__ float mean_resolution(float m6, float m7, float m9, float m10) {
    return __fmul_rn(__fadd_rn(hypot_fused(m6, m9), hypot_fused(m7, m10)), 0.5f);
}

// Fill entry `l` of a level table (block_m = float(4^l) * resolution).
__device__ __forceinline__ void fill_level(LevelTable &table, int l, float resolution,
                                           int4 cells) {
    const float block_m = __fmul_rn(static_cast<float>(1 << (2 * l)), resolution);
    const float step_km = __fmul_rn(block_m, 0.001f);
    table.side[l] = block_m;
    table.fallback[l] = __fmul_rn(__fmul_rn(block_m, 0.5f), 0.001f);
    table.out_step[l] = 0.001f > step_km ? 0.001f : step_km;
    // w carries the fallback's bits: a visit reads its cells and its
    // fallback with one 16-byte load.
    table.cells[l] = make_int4(cells.x, cells.y, cells.z, __float_as_int(table.fallback[l]));
}

// 2^shift as a float (exact; shift <= 38), from the exponent bits.
__device__ __forceinline__ float power_of_two(int shift) {
    return __int_as_float((127 + shift) << 23);
}

// Two FP32 lanes per instruction (the f32x2 operations of sm_100): each
// lane rounds exactly as the scalar __fadd_rn / __fmul_rn / __fmaf_rn does, so
// the march pairs its x and y arithmetic without changing a bit.
__device__ __forceinline__ float2 pair(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(reinterpret_cast<unsigned long long &>(d))
        : "l"(reinterpret_cast<const unsigned long long &>(a)),
          "l"(reinterpret_cast<const unsigned long long &>(b)));
    return d;
}

// The quartic path polynomial of both axes at once: lane x with
// (start_x, a1..a4), lane y with (start_y, b1..b4); d2, d3, d4 are the powers
// of the path offset d (cuda_backend.py:62-73).
__device__ __forceinline__ float2 quartic2(float2 x0, float2 k1, float2 k2, float2 k3,
                                           float2 k4, float2 d, float2 d2, float2 d3,
                                           float2 d4) {
    float2 r = __ffma2_rn(k1, d, x0);
    r = __ffma2_rn(k2, d2, r);
    r = __ffma2_rn(k3, d3, r);
    return __ffma2_rn(k4, d4, r);
}

// The Newton reciprocal of both lanes without the range fallback (the
// caller handles |x| >= 2^64).
__device__ __forceinline__ float2 newton_reciprocal_pair(float2 x) {
    const float2 y = pair(rcp_approx(x.x), rcp_approx(x.y));
    const float2 e = __ffma2_rn(__fmul2_rn(x, pair(-1.0f, -1.0f)), y, pair(1.0f, 1.0f));
    return __ffma2_rn(y, e, y);
}

// The correctly rounded reciprocal of both lanes (see rcp_approx), the
// Newton step issued as f32x2 pairs; each lane needs |x| >= 2^-64.  The
// march inlines the same choice with one branch for both lanes.
__device__ __forceinline__ float2 reciprocal_pair(float2 x) {
    float2 y = newton_reciprocal_pair(x);
    if (!(fabsf(x.x) < 0x1p64f)) y.x = __frcp_rn(x.x);
    if (!(fabsf(x.y) < 0x1p64f)) y.y = __frcp_rn(x.y);
    return y;
}

// Its derivative: a1 + 2 a2 d + 3 a3 d^2 + 4 a4 d^3 per lane
// (cuda_backend.py:76-84).
__device__ __forceinline__ float2 quartic_tangent2(float2 k1, float2 k2, float2 k3, float2 k4,
                                                   float2 d, float2 d2, float2 d3) {
    float2 r = __ffma2_rn(__fmul2_rn(pair(2.0f, 2.0f), k2), d, k1);
    r = __ffma2_rn(__fmul2_rn(pair(3.0f, 3.0f), k3), d2, r);
    return __ffma2_rn(__fmul2_rn(pair(4.0f, 4.0f), k4), d3, r);
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

// The relative arithmetic's level-0 sample: the height above `base` (the
// observer's z) at column origin_x + offset_x, row origin_y + offset_y.  The
// rounded absolute coordinates only decide the clamp; inside the clamp range
// the cell comes from the origin plus the offset's integer part and the
// fraction from the offset, and the corners are taken relative to `base`
// before they are interpolated.  Returns false (no data) when a corner is
// invalid.
__device__ __forceinline__ bool bilinear_above(const float *__restrict__ cells, int width,
                                               int height, int origin_x, float offset_x,
                                               float absolute_x, int origin_y, float offset_y,
                                               float absolute_y, float base, float &above) {
    const float cmax = __fsub_rn(static_cast<float>(width), 1.0001f);
    const float rmax = __fsub_rn(static_cast<float>(height), 1.0001f);
    int x0, y0;
    float tx, ty;
    if (absolute_x >= 0.0f && absolute_x <= cmax && absolute_y >= 0.0f && absolute_y <= rmax) {
        const float fx = floorf(offset_x), fy = floorf(offset_y);
        x0 = origin_x + static_cast<int>(fx);
        y0 = origin_y + static_cast<int>(fy);
        tx = __fsub_rn(offset_x, fx);
        ty = __fsub_rn(offset_y, fy);
    } else {
        float column = absolute_x > 0.0f ? absolute_x : 0.0f;
        column = column < cmax ? column : cmax;
        float row = absolute_y > 0.0f ? absolute_y : 0.0f;
        row = row < rmax ? row : rmax;
        x0 = static_cast<int>(floorf(column));
        y0 = static_cast<int>(floorf(row));
        tx = __fsub_rn(column, static_cast<float>(x0));
        ty = __fsub_rn(row, static_cast<float>(y0));
    }
    const int x1 = min(x0 + 1, width - 1);
    const int y1 = min(y0 + 1, height - 1);
    const float *r0 = cells + static_cast<size_t>(y0) * width;
    const float *r1 = cells + static_cast<size_t>(y1) * width;
    float q00 = __ldg(r0 + x0), q10 = __ldg(r0 + x1);
    float q01 = __ldg(r1 + x0), q11 = __ldg(r1 + x1);
    if (!(q00 > -20000.0f && q10 > -20000.0f && q01 > -20000.0f && q11 > -20000.0f))
        return false;
    q00 = __fsub_rn(q00, base);
    q10 = __fsub_rn(q10, base);
    q01 = __fsub_rn(q01, base);
    q11 = __fsub_rn(q11, base);
    const float top = __fmaf_rn(tx, __fsub_rn(q10, q00), q00);
    const float bottom = __fmaf_rn(tx, __fsub_rn(q11, q01), q01);
    above = __fmaf_rn(ty, __fsub_rn(bottom, top), top);
    return true;
}

// The relative arithmetic's far-field slope of a sample `above` metres above
// the observer's z: the four-cell bound's local-z formula (bound_slope) with
// the height difference given directly.
__device__ __forceinline__ float above_slope(float dist, float above, float radius,
                                             float observer_z, float observer_radius) {
    const float squared = __fmul_rn(dist, dist);
    float radius_sum = __fadd_rn(__fmul_rn(2.0f, radius), __fadd_rn(observer_z, above));
    radius_sum = __fadd_rn(radius_sum, observer_z);
    const float numerator = __fmaf_rn(above, radius_sum, -squared);
    const float local_z = __fdiv_rn(numerator, __fmul_rn(2.0f, observer_radius));
    const float lx2 = __fmaf_rn(-local_z, local_z, squared);
    const float local_x = lx2 > 0.0f ? __fsqrt_rn(lx2) : 1e-6f;
    return __fdiv_rn(local_z, local_x);
}

// Local-z slope of a terrain point seen over the chord `dist`
// (cuda_backend.py:812-830): numerator fused on its first product, local_x^2
// = dist*dist - local_z^2 fused on local_z*local_z (dist*dist rounded), as
// the reference's Numba-CUDA kernel computes it on the B200.
__device__ __forceinline__ float sample_slope(float dist, float height, float radius,
                                              float observer_radius) {
    const float squared = __fmul_rn(dist, dist);
    const float point_radius = __fadd_rn(radius, height);
    const float radius_delta = __fsub_rn(point_radius, observer_radius);
    const float radius_sum = __fadd_rn(point_radius, observer_radius);
    const float numerator = __fmaf_rn(radius_delta, radius_sum, -squared);
    const float local_z = __fdiv_rn(numerator, __fmul_rn(2.0f, observer_radius));
    const float lx2 = __fmaf_rn(-local_z, local_z, squared);
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
    const float lx2 = __fmaf_rn(-local_z, local_z, squared);
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

// Four-cell bound of the level cell (cx, cy): the maximum of the cell and its
// right / lower / diagonal neighbours, -32000 standing in for a missing one.
__device__ __forceinline__ float four_cell_bound(const float *__restrict__ cells, int4 L,
                                                 int cx, int cy) {
    const int index = L.x + cy * L.y + cx;
    const bool has_right = cx + 1 < L.y, has_down = cy + 1 < L.z;
    const float v00 = __ldg(cells + index);
    const float v10 = has_right ? __ldg(cells + index + 1) : -32000.0f;
    const float v01 = has_down ? __ldg(cells + index + L.y) : -32000.0f;
    const float v11 = has_right && has_down ? __ldg(cells + index + L.y + 1) : -32000.0f;
    return fmaxf(fmaxf(v00, v10), fmaxf(v01, v11));
}

// The same value read from the precomputed bound table (one load per visit).
__device__ __forceinline__ float cell_bound(const float *__restrict__ bounds, int4 L, int cx,
                                            int cy) {
    return __ldg(bounds + L.x + cy * L.y + cx);
}

// Advance (km) to the exit of the cell (cx, cy) of side 4^level pixels along
// the tangent, or `fallback` when the exit is not ahead, + 1e-4 km
// (cuda_backend.py:733-762).  Of max(t1, t2) only the far edge can win:
// (min_x - px) <= 0 < (max_x - px), so the product with inv_x keeps that
// order's sign pattern and the larger t is the edge ahead of the ray
// (bitwise the same value, including the -0.0 of a ray starting on the edge).
// (ux, uy) is the position relative to the integer origin (origin_x,
// origin_y); the reference arithmetic is origin 0 with u the absolute position.
__device__ __forceinline__ float cell_exit_advance(int shift, int cx, int cy, float ux, float uy,
                                                   int origin_x, int origin_y, float inv_x,
                                                   float inv_y, float fallback) {
    const float scale_f = power_of_two(shift);
    const float2 low = pair(static_cast<float>((cx << shift) - origin_x),
                            static_cast<float>((cy << shift) - origin_y));
    const float2 high = __fadd2_rn(low, pair(scale_f, scale_f));
    const float2 edge = pair(inv_x > 0.0f ? high.x : low.x, inv_y > 0.0f ? high.y : low.y);
    const float2 tm = __fmul2_rn(sub2(edge, pair(ux, uy)), pair(inv_x, inv_y));
    const float tmx = tm.x, tmy = tm.y;
    const float exit_distance = tmx < tmy ? tmx : tmy;
    // The reference returns `fallback` when the distance it adds 1e-4 km to
    // is not positive; that distance is the exit or, behind the ray, the
    // fallback, which is positive on every DEM that marches (the host
    // refuses pixel sizes too small for the ray length).  With a fallback of
    // zero the reference would not advance and its ray would never end.
    return __fadd_rn(exit_distance > 0.0f ? exit_distance : fallback, 0.0001f);
}

// The skip ladder.  After a cull at `level`, climb to the ancestors of the
// cell while each is culled by a conservative test, and return the advance
// to the exit of the largest culled one (`advance` when none is).  Every
// ancestor of an in-range cell is in range.  The test bounds the slope of
// every sample the skip passes over: heights are <= the ancestor's four-cell
// bound h, distances lie in [d0, d1] with d0 = true_m (distance grows along
// the ray) and d1 = d0 + 1010 m per km of advance + 1 m (a chord never
// outgrows the path).  With dh = h - observer_z >= 0 the slope falls with
// distance, so the bound is the slope formula at d0; with dh < 0 every slope
// is below dh / d1 (the curvature drop only lowers it).  The cull needs the
// bound below `current` by a relative 4e-6, which covers its rounding.
//
// The decision is made on a cheap approximation of the bound whenever it lies
// outside a guard band around `current` (as in bound_culled: the far-field
// approximation is within 2e-6 relative of the exact float32 bound, the
// divisions within 2 ulp; the band is 1e-5 relative), and with the exact
// arithmetic inside it, so the decision is always that of the exact test.
// ladder_culled tests the level-m ancestor and sets `step` to its exit
// advance; ladder_advance climbs from `level`, returns the advance and sets
// `reached` to the largest culled level (`level` if none).
template <class Table>
__device__ __forceinline__ bool ladder_culled(const Table &table, const float *__restrict__ bounds,
                                              int m, int ipx, int ipy, float ux, float uy,
                                              int origin_x, int origin_y,
                                              float inv_x, float inv_y, bool near, float true_m,
                                              float radius, float observer_z,
                                              float observer_radius, float inverse_denominator,
                                              float current, float &step) {
    const int shift = 2 * m;
    const int cx = ipx >> shift, cy = ipy >> shift;
    const int4 L = table.cells(m);
    const float maximum_height = cell_bound(bounds, L, cx, cy);
    step = cell_exit_advance(shift, cx, cy, ux, uy, origin_x, origin_y, inv_x, inv_y,
                             __int_as_float(L.w));
    if (maximum_height < -20000.0f) return true;
    const float dh = __fsub_rn(maximum_height, observer_z);
    const float far_distance = __fadd_rn(__fadd_rn(true_m, __fmul_rn(step, 1010.0f)), 1.0f);
    float approx;
    bool exact = false;
    if (dh < 0.0f) {
        approx = __fdividef(dh, far_distance);
    } else if (near) {
        approx = __fdividef(dh, true_m);
    } else {
        const float squared = __fmul_rn(true_m, true_m);
        float radius_sum = __fadd_rn(__fmul_rn(2.0f, radius), maximum_height);
        radius_sum = __fadd_rn(radius_sum, observer_z);
        const float numerator = __fmaf_rn(dh, radius_sum, -squared);
        const float local_z = __fmul_rn(numerator, inverse_denominator);
        const float lx2 = __fmaf_rn(true_m, true_m, -__fmul_rn(local_z, local_z));
        exact = !(lx2 > 0.25f * squared);
        approx = exact ? 0.0f : __fmul_rn(local_z, rsqrtf(lx2));
    }
    if (!exact) {
        const float size = fmaxf(fabsf(approx), fabsf(current));
        const float decided = __fadd_rn(approx, __fmul_rn(4e-6f, size));
        const float band = 1e-5f * size + 1e-30f;
        if (decided < current - band) return true;
        if (decided > current + band) return false;
    }
    float bound;
    if (dh < 0.0f) {
        bound = __fdiv_rn(dh, far_distance);
    } else {
        bound = near ? __fdiv_rn(dh, true_m)
                     : bound_slope(true_m, maximum_height, radius, observer_z, observer_radius);
    }
    const float size = fmaxf(fabsf(bound), fabsf(current));
    return __fadd_rn(bound, __fmul_rn(4e-6f, size)) <= current;
}

template <bool kCount, class Table>
__device__ __forceinline__ float ladder_advance(const Table &table, const float *__restrict__ bounds,
                                                int level, int top, int ipx, int ipy, float ux,
                                                float uy, int origin_x, int origin_y,
                                                float inv_x, float inv_y, bool near,
                                                float true_m, float radius, float observer_z,
                                                float observer_radius, float inverse_denominator,
                                                float current, float advance, unsigned &visits,
                                                int &reached) {
    reached = level;
    if (true_m < kLadderMinimumDistance) return advance;
    float best = advance;
    for (int m = level + 1; m <= top; ++m) {
        float step;
        if (kCount) ++visits;
        if (!ladder_culled(table, bounds, m, ipx, ipy, ux, uy, origin_x, origin_y, inv_x, inv_y,
                           near, true_m, radius, observer_z, observer_radius,
                           inverse_denominator, current, step))
            break;
        best = step;
        reached = m;
    }
    return best;
}

// One interpolated segment (fields 0,1,4..17 of the reference layout).
// With the relative arithmetic start_x, start_y are relative to the integer
// origin (origin_x, origin_y); otherwise the origin is 0.
struct RaySegment {
    float2 start;           // (start_x, start_y)
    float2 k1, k2, k3, k4;  // (a1, b1) .. (a4, b4)
    float s_start, s_end, s_start_chord, c1, c2, c3;
    int origin_x, origin_y;
};

// Subpatch interpolation of one ray's segment (cuda_backend.py:1032-1119):
// four centres around the pixel, their start points shifted to the pixel.
// kRelative: the origin is the integer part of the upper-left centre's start,
// and the four starts are taken relative to it before the shift and the
// interpolation (exact: they lie within a few pixels of each other).
template <bool kRelative = false>
__device__ __forceinline__ RaySegment interpolate_segment(
    const float *__restrict__ segments, int center_count, int dem_count, int pass_index,
    int azimuth, int column, int row, int tile_column, int tile_row, int tile_width,
    int subpatch, int primary_width, int primary_height, float ratio) {
    const int count = tile_width / subpatch + 2;
    const float gx = __fadd_rn(__fdiv_rn(static_cast<float>(column - subpatch / 2),
                                         static_cast<float>(subpatch)), 1.0f);
    const float gy = __fadd_rn(__fdiv_rn(static_cast<float>(row - subpatch / 2),
                                         static_cast<float>(subpatch)), 1.0f);
    int left = static_cast<int>(gx), top = static_cast<int>(gy);
    float tx = __fsub_rn(gx, static_cast<float>(left));
    float ty = __fsub_rn(gy, static_cast<float>(top));
    if (left < 0) { left = 0; tx = 0.0f; }
    if (top < 0) { top = 0; ty = 0.0f; }
    if (left > count - 2) { left = count - 2; tx = 1.0f; }
    if (top > count - 2) { top = count - 2; ty = 1.0f; }
    const int i00 = top * count + left, i10 = i00 + 1;
    const int i01 = (top + 1) * count + left, i11 = i01 + 1;
    const int req_left = tile_column + (left - 1) * subpatch + subpatch / 2;
    const int req_top = tile_row + (top - 1) * subpatch + subpatch / 2;
    const float d_left = static_cast<float>(
        column - (clamp_center(req_left, primary_width, subpatch) - tile_column));
    const float d_right = static_cast<float>(
        column - (clamp_center(req_left + subpatch, primary_width, subpatch) - tile_column));
    const float d_top = static_cast<float>(
        row - (clamp_center(req_top, primary_height, subpatch) - tile_row));
    const float d_bottom = static_cast<float>(
        row - (clamp_center(req_top + subpatch, primary_height, subpatch) - tile_row));

    const size_t stride_c = static_cast<size_t>(dem_count) * kSegmentFields;
    const float *base = segments + static_cast<size_t>(azimuth) * center_count * stride_c +
                        static_cast<size_t>(pass_index) * kSegmentFields;
    const float *s00 = base + i00 * stride_c, *s10 = base + i10 * stride_c;
    const float *s01 = base + i01 * stride_c, *s11 = base + i11 * stride_c;
    float seg[kMarchFields];
    int origin[2] = {0, 0};
    if (kRelative) {
        origin[0] = static_cast<int>(floorf(__ldg(s00 + 0)));
        origin[1] = static_cast<int>(floorf(__ldg(s00 + 1)));
    }
#pragma unroll
    for (int k = 0; k < kMarchFields; ++k) {
        const int f = k < 2 ? k : k + 2;
        float v00 = __ldg(s00 + f), v10 = __ldg(s10 + f);
        float v01 = __ldg(s01 + f), v11 = __ldg(s11 + f);
        if (kRelative && f < 2) {
            const float o = static_cast<float>(origin[f]);
            v00 = __fsub_rn(v00, o);
            v10 = __fsub_rn(v10, o);
            v01 = __fsub_rn(v01, o);
            v11 = __fsub_rn(v11, o);
        }
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
    return RaySegment{pair(seg[0], seg[1]), pair(seg[2], seg[6]), pair(seg[3], seg[7]),
                      pair(seg[4], seg[8]), pair(seg[5], seg[9]), seg[10], seg[11],
                      seg[12], seg[13], seg[14], seg[15], origin[0], origin[1]};
}

// The state of one ray within one DEM pass of hierarchy_maximum.
struct MarchState {
    float s;            // path position (km)
    float current;      // maximum slope so far (-1e30 for none)
    int level_hint;     // level of the previous step
    // side(level_hint + 1) (NaN at the top level) and side(level_hint)
    // (-inf at level 0): the level search keeps level_hint whenever
    // !(side_up <= footprint) && side_here <= footprint.
    float side_up, side_here;
};

// side_here = +inf sends the first step through the full level search.
__device__ __forceinline__ MarchState begin_pass(const DemView &dem, const RaySegment &g,
                                                 float current) {
    return MarchState{g.s_start > 0.001f ? g.s_start : 0.001f, current, dem.level_count - 1,
                      __int_as_float(0x7fffffff), INFINITY};
}

// Traversals of march_step, a bit set: the reference's (0), the skip ladder
// (bit 0) and the relative arithmetic (bit 1).
enum Traversal { kReference = 0, kLadderClimb = 1, kRelative = 2 };

// Which level-0 sample set the running maximum: nothing (NoArgmax, the
// production kernels) or its position, distance and slope (Argmax, the
// checkpoint of the DEM adjoint; `pass` is set by the caller).
struct NoArgmax {
    __device__ __forceinline__ void record(float, float, float, float, bool) {}
};
struct Argmax {
    float px = 0.0f, py = 0.0f, true_m = 0.0f, slope = -1e30f;
    int near = 0, pass = -1;
    int current_pass = 0;
    __device__ __forceinline__ void record(float x, float y, float distance, float value,
                                           bool is_near) {
        px = x;
        py = y;
        true_m = distance;
        slope = value;
        near = is_near ? 1 : 0;
        pass = current_pass;
    }
};

// One outer iteration of hierarchy_maximum (cuda_backend.py:672-867): one ray
// position, the level descent (and with the ladder the climb) and the advance.
// Returns false, leaving `st` untouched, when the pass is over (past s_end,
// outside the DEM, or the cell left the level grid).
template <bool kCount, int kLadder, class Table, class Tracker>
__device__ __forceinline__ bool march_step_tracked(const Table &table, const DemView &dem,
                                                   const RaySegment &g, int pass_index,
                                                   float observer_z, MarchState &st,
                                                   unsigned &visits, unsigned &samples,
                                                   unsigned &steps, Tracker &tracker) {
    const float radius = dem.radius;
    const float resolution = dem.resolution;
    const float observer_radius = __fadd_rn(radius, observer_z);
    const float inverse_denominator = __frcp_rn(__fmul_rn(2.0f, observer_radius));
    const float *__restrict__ cells = dem.cells;
    const float minimum_step = __fmul_rn(__fmul_rn(0.5f, resolution), 0.001f);
    const float primary_far_step = __fmul_rn(__fmul_rn(0.8f, resolution), 0.001f);
    const float last_x = static_cast<float>(dem.width - 1);
    const float last_y = static_cast<float>(dem.height - 1);
    const int top_level = dem.level_count - 1;
    float s = st.s;
    float current = st.current;
    int level_hint = st.level_hint;
    float side_up = st.side_up, side_here = st.side_here;
    constexpr bool relative = (kLadder & kRelative) != 0;
    if (!(s <= g.s_end)) return false;
    {
        if (kCount) ++steps;
        const float delta = __fsub_rn(s, g.s_start);
        const float2 d1 = pair(delta, delta);
        const float2 d2 = __fmul2_rn(d1, d1);
        const float2 d3 = __fmul2_rn(d2, d1);
        const float2 d4 = __fmul2_rn(d2, d2);
        // Relative arithmetic: offsets along the ray without the start, added
        // to the start relative to the origin; the absolute position (origin
        // + offset, rounded) only takes the bounds decisions.
        float2 r, u, p;
        if (relative) {
            r = quartic2(pair(0.0f, 0.0f), g.k1, g.k2, g.k3, g.k4, d1, d2, d3, d4);
            u = __fadd2_rn(g.start, r);
            p = __fadd2_rn(pair(static_cast<float>(g.origin_x), static_cast<float>(g.origin_y)),
                           u);
        } else {
            p = quartic2(g.start, g.k1, g.k2, g.k3, g.k4, d1, d2, d3, d4);
            u = p;
        }
        const float ux = u.x, uy = u.y, px = p.x, py = p.y;
        // NaN fails every comparison, as the reference's isnan tests do.
        if (!(px >= 0.0f && py >= 0.0f && px < last_x && py < last_y)) return false;
        const bool near = s < 0.5f;
        float true_m;
        if (near) {
            true_m = __fmul_rn(s, 1000.0f);
        } else {
            // The planar distance only feeds the far-field chord.
            if (!relative) r = sub2(p, g.start);
            const float2 planar = __fmul2_rn(r, pair(resolution, resolution));
            const float planar_m = hypot_fused(planar.x, planar.y);
            const float pm2 = __fmul_rn(planar_m, planar_m);
            // (c2 * pm2, pm2 * planar_m) in one instruction.
            const float2 terms = __fmul2_rn(pair(g.c2, pm2), pair(pm2, planar_m));
            float chord = __fmaf_rn(g.c1, planar_m, terms.x);
            chord = __fmaf_rn(g.c3, terms.y, chord);
            true_m = __fmaf_rn(g.s_start_chord, 1000.0f, chord);
        }
        const float footprint = __fmul_rn(true_m, 0.004363323129985824f);
        // The reference scans down from the top level to the largest level
        // whose side fits the footprint (or 0).  Sides grow with the level,
        // so that level is also found by moving up or down from the previous
        // step's level, which usually takes one comparison.
        // The two sides around the previous level sit in registers, so the
        // usual step decides with two comparisons and no table read.
        int level = level_hint;
        if (side_up <= footprint || !(side_here <= footprint)) {
            while (level < top_level && table.side(level + 1) <= footprint) ++level;
            while (level > 0 && !(table.side(level) <= footprint)) --level;
            level_hint = level;
            side_up = level < top_level ? table.side(level + 1) : __int_as_float(0x7fffffff);
            side_here = level > 0 ? table.side(level) : -INFINITY;
        }
        // The tangent and its reciprocals depend only on delta.
        const float2 tangent = quartic_tangent2(g.k1, g.k2, g.k3, g.k4, d1, d2, d3);
        const float dx = tangent.x, dy = tangent.y;
        // The Newton reciprocal is exact for 2^-64 <= |d| < 2^64 and used only
        // for |d| > 1e-8; a tangent of 2^64 or more (or not finite) takes the
        // IEEE reciprocal on a branch of its own.
        const float2 newton = newton_reciprocal_pair(tangent);
        const float ax = fabsf(dx), ay = fabsf(dy);
        float inv_x = ax > 1e-8f ? newton.x : 1e30f;
        float inv_y = ay > 1e-8f ? newton.y : 1e30f;
        if (!(ax < 0x1p64f && ay < 0x1p64f)) {
            inv_x = ax > 1e-8f ? __frcp_rn(dx) : 1e30f;
            inv_y = ay > 1e-8f ? __frcp_rn(dy) : 1e30f;
        }
        const int origin_x = relative ? g.origin_x : 0;
        const int origin_y = relative ? g.origin_y : 0;
        const int ipx = relative ? origin_x + static_cast<int>(floorf(ux)) : static_cast<int>(px);
        const int ipy = relative ? origin_y + static_cast<int>(floorf(uy)) : static_cast<int>(py);
        bool ray_out = false;
        for (;;) {
            const int4 L = table.cells(level);
            const int shift = level * 2;
            const int cx = ipx >> shift, cy = ipy >> shift;
            if (kCount) ++visits;
            if (cx >= L.y || cy >= L.z) {  // cx, cy >= 0 since px, py >= 0
                s = __fadd_rn(s, table.out_step(level));
                ray_out = true;
                break;
            }
            const float maximum_height = cell_bound(dem.bounds, L, cx, cy);
            const float skip = cell_exit_advance(shift, cx, cy, ux, uy, origin_x, origin_y, inv_x,
                                                 inv_y, __int_as_float(L.w));
            bool culled = maximum_height < -20000.0f;
            if (!culled) {
                const float scale_f = power_of_two(shift);
                float true_near = __fmaf_rn(-scale_f, resolution, true_m);
                true_near = true_near > 1.0f ? true_near : 1.0f;
                culled = bound_culled(near, true_near, maximum_height, radius, observer_z,
                                      observer_radius, inverse_denominator, current);
            }
            if (culled) {
                float advance = skip;
                if (kLadder & kLadderClimb) {
                    int reached;
                    advance = ladder_advance<kCount>(table, dem.bounds, level, top_level, ipx, ipy,
                                                     ux, uy, origin_x, origin_y, inv_x, inv_y,
                                                     near, true_m, radius, observer_z,
                                                     observer_radius, inverse_denominator,
                                                     current, skip, visits, reached);
                }
                s = __fadd_rn(s, advance);
                break;
            }
            if (level == 0) {
                if (kCount) ++samples;
                float slope = -1e30f;
                if (relative) {
                    float above;
                    if (bilinear_above(cells, dem.width, dem.height, origin_x, ux, px, origin_y,
                                       uy, py, observer_z, above)) {
                        slope = near ? __fdiv_rn(above, true_m)
                                     : above_slope(true_m, above, radius, observer_z,
                                                   observer_radius);
                        if (slope > current) {
                            current = slope;
                            tracker.record(px, py, true_m, slope, near);
                        }
                    }
                } else {
                    const float height = bilinear(cells, dem.width, dem.height, px, py);
                    if (height > -20000.0f) {
                        slope = near ? __fdiv_rn(__fsub_rn(height, observer_z), true_m)
                                     : sample_slope(true_m, height, radius, observer_radius);
                        if (slope > current) {
                            current = slope;
                            tracker.record(px, py, true_m, slope, near);
                        }
                    }
                }
                const float magnitude = hypot_fused(dx, dy);
                const float pixel_step = magnitude > 1e-6f ? __frcp_rn(magnitude) : 0.0005f;
                // inner = min(margin_step, angular_step), both a product
                // divided by 1000 (the margin one 0 unless margin > 0).  A
                // correctly rounded division by a positive constant is
                // monotone, so the smaller quotient is the quotient of the
                // smaller product: one division gives the same value.
                const float margin = __fsub_rn(current, slope);
                const float angular_product = __fmul_rn(true_m, 0.00151f);
                float inner = 0.0f;
                if (margin > 0.0f) {
                    const float margin_product = __fmul_rn(__fmul_rn(margin, true_m), 1.732f);
                    inner = __fdiv_rn(margin_product < angular_product ? margin_product
                                                                       : angular_product,
                                      1000.0f);
                }
                float advance = pixel_step > inner ? pixel_step : inner;
                if (near) advance = __fmul_rn(advance, 0.25f);
                const float floor_step =
                    (pass_index == 0 && true_m >= 100.0f) ? primary_far_step : minimum_step;
                advance = advance > floor_step ? advance : floor_step;
                s = __fadd_rn(s, advance);
                break;
            }
            --level;
        }
        if (ray_out) return false;
    }
    st.s = s;
    st.current = current;
    st.level_hint = level_hint;
    st.side_up = side_up;
    st.side_here = side_here;
    return true;
}

// hierarchy_maximum (cuda_backend.py:656-874): the maximum slope along one
// ray over one DEM, starting from `current` (-1e30 for none).  Table gives
// side(l), fallback(l), out_step(l) and cells(l).
template <bool kCount, int kLadder, class Table>
__device__ __forceinline__ bool march_step(const Table &table, const DemView &dem,
                                           const RaySegment &g, int pass_index,
                                           float observer_z, MarchState &st, unsigned &visits,
                                           unsigned &samples, unsigned &steps) {
    NoArgmax none;
    return march_step_tracked<kCount, kLadder>(table, dem, g, pass_index, observer_z, st,
                                               visits, samples, steps, none);
}

template <bool kCount, int kLadder, class Table, class Tracker>
__device__ __forceinline__ float march_dem_tracked(const Table &table, const DemView &dem,
                                                   const RaySegment &g, int pass_index,
                                                   float observer_z, float current,
                                                   unsigned &visits, unsigned &samples,
                                                   unsigned &steps, Tracker &tracker) {
    MarchState st = begin_pass(dem, g, current);
    while (march_step_tracked<kCount, kLadder>(table, dem, g, pass_index, observer_z, st,
                                               visits, samples, steps, tracker)) {
    }
    return st.current;
}

template <bool kCount, int kLadder, class Table>
__device__ __forceinline__ float march_dem(const Table &table, const DemView &dem,
                                           const RaySegment &g, int pass_index,
                                           float observer_z, float current, unsigned &visits,
                                           unsigned &samples, unsigned &steps) {
    NoArgmax none;
    return march_dem_tracked<kCount, kLadder>(table, dem, g, pass_index, observer_z, current,
                                              visits, samples, steps, none);
}

}  // namespace ls200
