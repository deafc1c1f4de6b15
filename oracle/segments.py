"""ORACLE — test infrastructure only.  Ray-segment tensor generation.

Restates the host side of src/lunarscout/_numba_horizon/geometry.py:
``inverse_stereographic`` :153-182, ``lat_lon_to_vector`` :197-208,
``enu_to_moon_matrix`` :219-226, ``azimuth_direction`` :229-234,
``DemGrid.elevation`` :98-110, ``build_dem_segment_contexts`` :452-462,
``clamp_subpatch_center``/``build_subpatch_centers`` :465-487 and
``build_subpatch_segments_numba`` :575-673.  The per-job chord sampling and
fitting runs in ``segments.c``.

DEM arguments are duck-typed: ``elevation_m`` float32[y, x], ``geo_transform``
float64[6] and ``projection`` with ``radius_m``, ``latitude_origin_rad``,
``longitude_origin_rad``, ``scale``, ``false_easting_m``, ``false_northing_m``.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _declare_extra, default_threads, lib

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_declare_extra(
    "ora_segments_dem",
    [_f32p, ctypes.c_int, ctypes.c_int, _f64p, _f64p, _f64p, _f64p, _f64p,
     ctypes.c_double, ctypes.c_double, _f64p, ctypes.c_longlong, _f32p, ctypes.c_int],
    ctypes.c_int,
)
_declare_extra(
    "ora_segment_samples",
    [_f32p, ctypes.c_int, ctypes.c_int, _f64p, _f64p, _f64p, _f64p,
     ctypes.c_double, ctypes.c_double, _f64p],
    ctypes.c_int,
)


def projection_array(dem) -> np.ndarray:
    p = dem.projection
    return np.array(
        (p.radius_m, p.latitude_origin_rad, p.longitude_origin_rad, p.scale,
         p.false_easting_m, p.false_northing_m),
        dtype=np.float64,
    )


def map_resolution_m(dem) -> float:
    t = dem.geo_transform
    return float((math.hypot(t[1], t[4]) + math.hypot(t[2], t[5])) * 0.5)


def pixel_to_crs(dem, column: float, row: float) -> tuple[float, float]:
    t = dem.geo_transform
    return (
        float(t[0] + t[1] * column + t[2] * row),
        float(t[3] + t[4] * column + t[5] * row),
    )


def inverse_stereographic(x: float, y: float, p) -> tuple[float, float]:
    xp = x - p.false_easting_m
    yp = y - p.false_northing_m
    rho = math.hypot(xp, yp)
    if rho < 1e-9:
        return p.latitude_origin_rad, p.longitude_origin_rad
    c = 2.0 * math.atan2(rho, 2.0 * p.scale * p.radius_m)
    sin_c, cos_c = math.sin(c), math.cos(c)
    sin_o, cos_o = math.sin(p.latitude_origin_rad), math.cos(p.latitude_origin_rad)
    latitude = math.asin(cos_c * sin_o + yp * sin_c * cos_o / rho)
    longitude = p.longitude_origin_rad + math.atan2(
        xp * sin_c, rho * cos_o * cos_c - yp * sin_o * sin_c
    )
    return latitude, longitude


def dem_elevation(dem, column: float, row: float) -> float:
    """FP64 bilinear of ``DemGrid.elevation`` (no clamping, no validity)."""
    e = dem.elevation_m
    height, width = e.shape
    x1, y1 = int(column), int(row)
    x2, y2 = min(x1 + 1, width - 1), min(y1 + 1, height - 1)
    q11, q12 = float(e[y1, x1]), float(e[y2, x1])
    q21, q22 = float(e[y1, x2]), float(e[y2, x2])
    return (
        q11 * (x2 - column) * (y2 - row)
        + q21 * (column - x1) * (y2 - row)
        + q12 * (x2 - column) * (row - y1)
        + q22 * (column - x1) * (row - y1)
    )


def enu_rows(latitude: float, longitude: float) -> tuple[tuple, tuple, tuple]:
    cos_lat, sin_lat = math.cos(latitude), math.sin(latitude)
    cos_lon, sin_lon = math.cos(longitude), math.sin(longitude)
    east = (-sin_lon, cos_lon, 0.0)
    north = (-sin_lat * cos_lon, -sin_lat * sin_lon, cos_lat)
    up = (cos_lat * cos_lon, cos_lat * sin_lon, sin_lat)
    return east, north, up


def azimuth_directions(latitude: float, longitude: float, azimuth_count: int) -> np.ndarray:
    """Unit Moon-centred direction of each azimuth (0 = north, clockwise)."""
    east, north, _up = enu_rows(latitude, longitude)
    out = np.empty((azimuth_count, 3), dtype=np.float64)
    for index in range(azimuth_count):
        angle = math.pi / 2.0 - index * 2.0 * math.pi / azimuth_count
        c, s = math.cos(angle), math.sin(angle)
        d = [c * east[k] + s * north[k] for k in range(3)]
        norm = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        out[index] = (d[0] / norm, d[1] / norm, d[2] / norm)
    return out


def clamp_center(requested: int, dem_size: int, subpatch: int) -> int:
    half = subpatch // 2
    return min(max(requested, half), max(half, dem_size - half))


def subpatch_centers(tile_column, tile_row, tile_width, subpatch, width, height):
    """(requested, clamped) centre per subpatch index, row-major."""
    count = tile_width // subpatch + 2
    centers = []
    for index in range(count * count):
        grid_row, grid_column = divmod(index, count)
        rc = tile_column + (grid_column - 1) * subpatch + subpatch // 2
        rr = tile_row + (grid_row - 1) * subpatch + subpatch // 2
        centers.append(
            (clamp_center(rc, width, subpatch), clamp_center(rr, height, subpatch))
        )
    return centers


def segment_jobs(dems, *, tile_column, tile_row, tile_width, azimuth_count,
                 observer_elevation_m, subpatch_size):
    """Unique centres, their observers/radii and per-(centre, azimuth) directions."""
    primary = dems[0]
    height, width = primary.elevation_m.shape
    centers = subpatch_centers(tile_column, tile_row, tile_width, subpatch_size, width, height)
    unique = list(dict.fromkeys(centers))
    observers = np.empty((len(unique), 3), dtype=np.float64)
    radii = np.empty(len(unique), dtype=np.float64)
    directions = np.empty((len(unique), azimuth_count, 3), dtype=np.float64)
    for index, (cc, cr) in enumerate(unique):
        x, y = pixel_to_crs(primary, cc, cr)
        latitude, longitude = inverse_stereographic(x, y, primary.projection)
        tc = min(max(float(cc), 0.0), width - 1.001)
        tr = min(max(float(cr), 0.0), height - 1.001)
        terrain = dem_elevation(primary, tc, tr)
        radii[index] = primary.projection.radius_m + terrain
        r = radii[index] + observer_elevation_m
        cos_lat = math.cos(latitude)
        observers[index] = (
            r * cos_lat * math.cos(longitude),
            r * cos_lat * math.sin(longitude),
            r * math.sin(latitude),
        )
        directions[index] = azimuth_directions(latitude, longitude, azimuth_count)
    return centers, unique, observers, radii, directions


def build_segments(
    dems, *, tile_column: int, tile_row: int, tile_width: int = 128,
    azimuth_count: int = 1440, maximum_distance_m: float = 1_000_000.0,
    observer_elevation_m: float = 0.0, subpatch_size: int = 8,
    threads: int | None = None,
) -> np.ndarray:
    """Dense segment tensor float32[A, C, D, 18] (geometry.py:575-673)."""
    dems = tuple(dems)
    centers, unique, observers, radii, directions = segment_jobs(
        dems, tile_column=tile_column, tile_row=tile_row, tile_width=tile_width,
        azimuth_count=azimuth_count, observer_elevation_m=observer_elevation_m,
        subpatch_size=subpatch_size,
    )
    job_count = len(unique) * azimuth_count
    job_observers = np.ascontiguousarray(np.repeat(observers, azimuth_count, axis=0))
    job_directions = np.ascontiguousarray(directions.reshape(job_count, 3))
    job_radii = np.ascontiguousarray(np.repeat(radii, azimuth_count))
    starts = np.ones(job_count, dtype=np.float64)
    unique_result = np.zeros((azimuth_count, len(unique), len(dems), 18), dtype=np.float32)
    for dem_index, dem in enumerate(dems):
        resolution = map_resolution_m(dem)
        height, width = dem.elevation_m.shape
        size_m = min(width * resolution, height * resolution)
        ray_limit = min(maximum_distance_m, size_m * 1.2)
        active = np.flatnonzero(starts < maximum_distance_m)
        if not len(active):
            break
        fitted = np.empty((len(active), 18), dtype=np.float32)
        lib().ora_segments_dem(
            np.ascontiguousarray(dem.elevation_m, dtype=np.float32), width, height,
            np.ascontiguousarray(dem.geo_transform, dtype=np.float64),
            projection_array(dem),
            np.ascontiguousarray(job_observers[active]),
            np.ascontiguousarray(job_directions[active]),
            np.ascontiguousarray(starts[active]), float(ray_limit), float(resolution),
            np.ascontiguousarray(job_radii[active]), len(active), fitted,
            int(threads or default_threads()),
        )
        unique_result[active % azimuth_count, active // azimuth_count, dem_index] = fitted
        last = fitted[:, 13].astype(np.float64) * 1000.0
        starts[active] = np.minimum(ray_limit, last)
    index = {key: i for i, key in enumerate(unique)}
    result = np.empty((azimuth_count, len(centers), len(dems), 18), dtype=np.float32)
    for center_index, key in enumerate(centers):
        result[:, center_index] = unique_result[:, index[key]]
    return result
