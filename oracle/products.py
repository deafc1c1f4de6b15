"""ORACLE — test infrastructure only.  Lighting products on the CPU.

* ``lighting_tiles``: lightmap_cpu.py:25-183 (sun fraction / body margin),
  per-pixel arithmetic in lighting.c.
* ``psr_tile``: psr.py:94-140 (FP64 PSR, lighting.c).
* ``reduce_sun_vectors``: psr.py:61-91 (five viewpoints x 1440 bins).
* ``longest_duration``: mission_duration.py:164-256 (longest right-censored
  run per candidate-start interval) on a dense condition cube.
* ``encode_tile`` / ``decode_tile``: file_format.py:39-73, 135-182 (.cbin).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _declare_extra, default_threads, lib

AZ = 1440
PATCH = 128
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_c = ctypes

_declare_extra("ora_lighting_tile",
               [_f32p, _f64p, _f64p, _f32p, _c.c_int, _f32p, _c.c_int, _c.c_int, _c.c_int,
                _c.c_int, _c.c_int, _f32p, _c.c_int], _c.c_int)
_declare_extra("ora_half_circle", [_f32p, _c.c_void_p], _c.c_int)
_declare_extra("ora_sun_fraction", [_f32p, _f32p, _f32p, _c.c_int, _f32p], _c.c_int)


def sun_fraction(horizons, azimuth_deg, elevation_deg) -> np.ndarray:
    """Visible disk fraction per horizon row at float32 (azimuth, elevation)."""
    horizons = np.ascontiguousarray(horizons, dtype=np.float32).reshape(-1, AZ)
    n = len(horizons)
    az = np.ascontiguousarray(np.broadcast_to(np.asarray(azimuth_deg, np.float32), (n,)))
    el = np.ascontiguousarray(np.broadcast_to(np.asarray(elevation_deg, np.float32), (n,)))
    out = np.empty(n, dtype=np.float32)
    lib().ora_sun_fraction(horizons, az, el, n, out)
    return out
_declare_extra("ora_psr_tile",
               [_f32p, _c.c_int, _c.c_int, _f64p, _f64p, _f64p, _c.c_int, _f32p, _c.c_int,
                _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_double, _u8p, _c.c_int], _c.c_int)
_declare_extra("ora_psr_viewpoints",
               [_f32p, _c.c_int, _c.c_int, _f64p, _f64p, _f64p, _c.c_int, _f64p, _f64p],
               _c.c_int)

#: -float(float32(0.545)) / 2 (psr.py:12,119)
PSR_LIMB_THRESHOLD = -float(np.float32(0.545)) / 2.0


def _projection(dem) -> np.ndarray:
    p = dem.projection
    return np.array((p.radius_m, p.latitude_origin_rad, p.longitude_origin_rad, p.scale,
                     p.false_easting_m, p.false_northing_m), dtype=np.float64)


def half_circle() -> tuple[np.ndarray, float]:
    out = np.zeros(16, dtype=np.float32)
    photons = ctypes.c_float()
    lib().ora_half_circle(out, ctypes.addressof(photons))
    return out, float(photons.value)


def patch_dem(dem, tile_y, tile_x, valid_height, valid_width) -> np.ndarray:
    patch = np.zeros((PATCH, PATCH), dtype=np.float32)
    patch[:valid_height, :valid_width] = dem.elevation_m[tile_y:tile_y + valid_height,
                                                         tile_x:tile_x + valid_width]
    return patch


def lighting_tiles(dem, horizons_deg, vectors_m, *, tile_y, tile_x, valid_height=PATCH,
                   valid_width=PATCH, margin=False, threads=None) -> np.ndarray:
    """float32[T, valid_h, valid_w] sun fractions (or margins in degrees)."""
    vectors = np.ascontiguousarray(np.asarray(vectors_m, dtype=np.float64), dtype=np.float32)
    horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32).reshape(PATCH, PATCH, AZ)
    out = np.zeros((len(vectors), PATCH, PATCH), dtype=np.float32)
    lib().ora_lighting_tile(
        patch_dem(dem, tile_y, tile_x, valid_height, valid_width),
        np.ascontiguousarray(dem.geo_transform, dtype=np.float64), _projection(dem),
        vectors, len(vectors), horizons, tile_x, tile_y, valid_width, valid_height,
        1 if margin else 0, out, int(threads or default_threads()))
    return out[:, :valid_height, :valid_width]


def encode_fraction_bytes(fractions: np.ndarray) -> np.ndarray:
    """uint8(float32(255) * fraction) (lightmap_cpu.py:233-236)."""
    return (np.asarray(fractions, dtype=np.float32) * np.float32(255.0)).astype(np.uint8)


def psr_tile(dem, horizons_deg, vectors_m, *, tile_y, tile_x, valid_height=PATCH,
             valid_width=PATCH, threads=None) -> np.ndarray:
    horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
    if horizons.shape == (PATCH, PATCH, AZ):
        stride = PATCH
    else:
        horizons = horizons.reshape(valid_height, valid_width, AZ)
        stride = valid_width
    vectors = np.ascontiguousarray(vectors_m, dtype=np.float64)
    out = np.empty((valid_height, valid_width), dtype=np.uint8)
    lib().ora_psr_tile(
        np.ascontiguousarray(dem.elevation_m, dtype=np.float32), dem.elevation_m.shape[1],
        dem.elevation_m.shape[0], np.ascontiguousarray(dem.geo_transform, np.float64),
        _projection(dem), vectors, len(vectors), horizons, stride, tile_x, tile_y,
        valid_width, valid_height, PSR_LIMB_THRESHOLD, out, int(threads or default_threads()))
    return out


_declare_extra("ora_psr_peak",
               [_f32p, _c.c_int, _c.c_int, _f64p, _f64p, _f64p, _c.c_int, _f32p, _c.c_int,
                _c.c_int, _c.c_int, _c.c_int, _c.c_int, _f64p, _c.c_int], _c.c_int)


def psr_peak_margin(dem, horizons_deg, vectors_m, *, tile_y, tile_x, valid_height=PATCH,
                    valid_width=PATCH, threads=None) -> np.ndarray:
    """Per pixel max over vectors of (elevation - horizon), FP64 (deg)."""
    horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
    stride = PATCH if horizons.shape == (PATCH, PATCH, AZ) else valid_width
    vectors = np.ascontiguousarray(vectors_m, dtype=np.float64)
    out = np.empty((valid_height, valid_width), dtype=np.float64)
    lib().ora_psr_peak(
        np.ascontiguousarray(dem.elevation_m, dtype=np.float32), dem.elevation_m.shape[1],
        dem.elevation_m.shape[0], np.ascontiguousarray(dem.geo_transform, np.float64),
        _projection(dem), vectors, len(vectors), horizons, stride, tile_x, tile_y,
        valid_width, valid_height, out, int(threads or default_threads()))
    return out


def reduce_sun_vectors(dem, vectors_m) -> tuple[np.ndarray, np.ndarray]:
    """Keep, per viewpoint and 0.25-deg azimuth bin, the highest vector;
    dedupe in first-seen order (psr.py:61-91)."""
    vectors = np.ascontiguousarray(vectors_m, dtype=np.float64)
    count = len(vectors)
    azimuth = np.empty((5, count), dtype=np.float64)
    elevation = np.empty((5, count), dtype=np.float64)
    lib().ora_psr_viewpoints(
        np.ascontiguousarray(dem.elevation_m, dtype=np.float32), dem.elevation_m.shape[1],
        dem.elevation_m.shape[0], np.ascontiguousarray(dem.geo_transform, np.float64),
        _projection(dem), vectors, count, azimuth, elevation)
    selected = np.full((5, AZ), -1, dtype=np.int64)
    maxima = np.full((5, AZ), -np.inf, dtype=np.float64)
    for p in range(5):
        bins = (azimuth[p] * (AZ / 360.0)).astype(np.int64) % AZ
        for index, b in enumerate(bins):
            if elevation[p, index] > maxima[p, b]:
                maxima[p, b] = elevation[p, index]
                selected[p, b] = index
    order = []
    seen = set()
    for value in selected.ravel():
        value = int(value)
        if value >= 0 and value not in seen:
            seen.add(value)
            order.append(value)
    indices = np.asarray(order, dtype=np.int64)
    return np.ascontiguousarray(vectors[indices]), indices


def longest_duration(condition: np.ndarray, sample_hours: np.ndarray,
                     accepts: np.ndarray) -> np.ndarray:
    """Longest right-censored run per candidate interval.

    condition bool[T, H, W]; sample_hours f64[T] (duration credited to sample
    t); accepts bool[I, T] (sample t lies in interval i's start window).
    Returns f64[I, H, W] hours (mission_duration.py:212-256).
    """
    condition = np.asarray(condition, dtype=bool)
    count, height, width = condition.shape
    intervals = accepts.shape[0]
    active = np.zeros((intervals, height, width), dtype=bool)
    current = np.zeros((intervals, height, width), dtype=np.float64)
    longest = np.zeros((intervals, height, width), dtype=np.float64)
    has_active = np.zeros(intervals, dtype=bool)
    for t in range(count):
        c = condition[t]
        false_now = ~c
        for i in range(intervals):
            if not accepts[i, t] and not has_active[i]:
                continue
            band = active[i]
            ended = band & false_now
            if np.any(ended):
                longest[i][ended] = np.maximum(longest[i][ended], current[i][ended])
                current[i][ended] = 0.0
                band[ended] = False
            if accepts[i, t]:
                band |= c
            accruing = band & c
            current[i][accruing] += sample_hours[t]
            has_active[i] = np.any(band)
    return np.maximum(longest, current)


def safe_haven(fractions: np.ndarray, margins: np.ndarray, month_index_of: np.ndarray,
               band_count: int, *, sunlight_threshold: float, earth_threshold_deg: float,
               time_step_hours: float) -> np.ndarray:
    """Per-band safe-haven hours, float32[B, H, W] with NaN nodata
    (safe_haven.py:75-243), stepping through time as the reference does.

    fractions, margins float32[T, H, W]; month_index_of int32[T] (-1: none).
    Per step: the low-Sun run length grows or resets (:180); the step's band
    records an outage or not and marks the run when it is low-Sun during an
    outage (:184-189); every marked band takes the run length while the run
    lasts, and marks clear when it ends (:194-201).  Bands without an outage,
    or without a non-outage sample, are NaN (:231-240).
    """
    fractions = np.asarray(fractions, dtype=np.float32)
    margins = np.asarray(margins, dtype=np.float32)
    count, height, width = fractions.shape
    shape = (height, width)
    run = np.zeros(shape, dtype=np.int32)
    touching = np.zeros((band_count, *shape), dtype=bool)
    best = np.zeros((band_count, *shape), dtype=np.int32)
    outage_seen = np.zeros((band_count, *shape), dtype=bool)
    above_seen = np.zeros((band_count, *shape), dtype=bool)
    for t in range(count):
        low = fractions[t] < np.float32(sunlight_threshold)
        outage = margins[t] < np.float32(earth_threshold_deg)
        run = np.where(low, run + 1, 0).astype(np.int32)
        band = int(month_index_of[t])
        if band >= 0:
            above_seen[band] |= ~outage
            outage_seen[band] |= outage
            touching[band] |= outage & low
        for b in range(band_count):
            best[b] = np.maximum(best[b], np.where(touching[b] & low, run, 0))
            touching[b] &= low
    out = best.astype(np.float32) * np.float32(time_step_hours)
    out[~outage_seen | ~above_seen] = np.nan
    return out


def earth_visibility(margins: np.ndarray, threshold_deg: float = 0.0) -> np.ndarray:
    """Share of time steps with Earth margin >= threshold, float32[H, W]
    (count / T in FP64, rounded to float32), from float32[T, H, W] margins
    (lightmap_cpu.py:121-141 per step)."""
    margins = np.asarray(margins, dtype=np.float32)
    counts = np.count_nonzero(margins >= np.float32(threshold_deg), axis=0)
    return (counts.astype(np.float64) / margins.shape[0]).astype(np.float32)


_SHORT_SCALE = np.float32(32767.0) / np.float32(50.0)
_ELEVATION_SCALE = np.float32(50.0) / np.float32(32767.0)


def encode_tile(degrees: np.ndarray) -> bytes:
    """.cbin payload of a pixel-major float32[16384, 1440] tile."""
    degrees = np.asarray(degrees, dtype=np.float32).reshape(-1, AZ)
    clipped = np.clip(degrees.astype(np.float64), -50.0, 50.0)
    scaled = (clipped.astype(np.float32) * _SHORT_SCALE).astype(np.float64)
    quantized = np.where(scaled >= 0, np.floor(scaled + 0.5), np.ceil(scaled - 0.5))
    quantized = np.clip(quantized, -32767, 32767).astype(np.int64)
    out = bytearray()
    for row in quantized:
        block = bytearray()
        previous = int(row[0])
        block += bytes(((previous >> 8) & 0xFF, previous & 0xFF))
        for q in row[1:]:
            delta = max(-16384, min(16383, int(q) - previous))
            previous = ((previous + delta + 32768) % 65536) - 32768
            if 0 <= delta < 63:
                block.append(delta)
            elif -64 <= delta < 0:
                block.append(delta & 0x7F)
            else:
                block += bytes((((delta >> 8) & 0xFF) | 0x80, delta & 0xFF))
        out += len(block).to_bytes(2, "little") + block
    return bytes(out)


def decode_tile(payload: bytes) -> np.ndarray:
    data = np.frombuffer(payload, dtype=np.uint8)
    pixels = PATCH * PATCH
    out = np.empty((pixels, AZ), dtype=np.float32)
    offset = 0
    for p in range(pixels):
        length = int(data[offset]) | (int(data[offset + 1]) << 8)
        offset += 2
        end = offset + length
        acc = (int(data[offset]) << 8) | int(data[offset + 1])
        if acc >= 32768:
            acc -= 65536
        offset += 2
        out[p, 0] = np.float32(acc) * _ELEVATION_SCALE
        k = 1
        while offset < end and k < AZ:
            first = int(data[offset])
            offset += 1
            if first & 0x80:
                high = ((first << 1) & 0x80) | (first & 0x7F)
                delta = (high << 8) | int(data[offset])
                offset += 1
                if delta >= 32768:
                    delta -= 65536
            else:
                delta = first & 0x7F
                if delta & 0x40:
                    delta -= 0x80
            acc = ((acc + delta + 32768) % 65536) - 32768
            out[p, k] = np.float32(acc) * _ELEVATION_SCALE
            k += 1
        if k != AZ or offset != end:
            raise ValueError("compressed horizon block did not decode to 1440 samples")
    if offset != len(data):
        raise ValueError("compressed horizon contains trailing bytes")
    return out
