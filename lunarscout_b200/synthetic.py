"""Seeded synthetic lunar inputs for tests and benchmarks.

The reference benchmarks real LOLA DEMs that are not available here; these
generators stand in with the same shapes, sizes and value distributions:

* DEMs: spectral fBm (amplitude ~ k^-(H+1), Hurst H) rescaled to a target
  standard deviation, plus parabolic bowl craters with power-law diameters
  (pdf ~ D^-2), depth 0.2 D and a raised rim of 0.04 D, on a south-polar
  stereographic grid (R = 1 737 400 m) centred on a given latitude/longitude.
* Sun vectors in the Moon-ME frame at 1 AU with a sub-solar latitude of
  1.54 deg * sin(2 pi t / 346.6 d) and a sub-solar longitude that turns once
  per 29.53 d; Earth vectors at ~384 400 km with optical librations of
  +-6.7 deg (27.21 d) in latitude and +-7.9 deg (27.55 d) in longitude.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .contract import MOON_RADIUS_M, DemGrid, ProjectionParameters

AU_M = 149_597_870_700.0
EARTH_DISTANCE_M = 384_400_000.0


def project_south_polar(latitude_rad: float, longitude_rad: float,
                        projection: ProjectionParameters) -> tuple[float, float]:
    """Forward spherical stereographic projection (geometry.py:185-193)."""
    sin_lat, cos_lat = math.sin(latitude_rad), math.cos(latitude_rad)
    sin_o = math.sin(projection.latitude_origin_rad)
    cos_o = math.cos(projection.latitude_origin_rad)
    delta = longitude_rad - projection.longitude_origin_rad
    denominator = 1.0 + sin_o * sin_lat + cos_o * cos_lat * math.cos(delta)
    if abs(denominator) < 1e-10:
        denominator = 1e-10
    scale = 2.0 * projection.scale * projection.radius_m / denominator
    x = scale * cos_lat * math.sin(delta) + projection.false_easting_m
    y = scale * (cos_o * sin_lat - sin_o * cos_lat * math.cos(delta))
    return x, y + projection.false_northing_m


def fbm_surface(height: int, width: int, *, hurst: float, sigma_m: float,
                rng: np.random.Generator) -> np.ndarray:
    """Spectral-synthesis fBm with amplitude ~ k^-(H+1), zero mean, std sigma."""
    ky = np.fft.fftfreq(height)[:, None]
    kx = np.fft.rfftfreq(width)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amplitude = k ** (-(hurst + 1.0))
    amplitude[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, size=amplitude.shape)
    noise = rng.standard_normal(size=amplitude.shape)
    spectrum = amplitude * noise * np.exp(1j * phase)
    surface = np.fft.irfft2(spectrum, s=(height, width))
    surface -= surface.mean()
    std = surface.std()
    if std > 0:
        surface *= sigma_m / std
    return surface


def add_craters(surface: np.ndarray, resolution_m: float, count: int, *,
                min_diameter_m: float, max_diameter_m: float,
                rng: np.random.Generator) -> None:
    """Parabolic bowls: floor -0.2 D, rim +0.04 D at r = D/2, ejecta ~ r^-3."""
    height, width = surface.shape
    u = rng.uniform(0.0, 1.0, size=count)
    inverse_min, inverse_max = 1.0 / min_diameter_m, 1.0 / max_diameter_m
    diameters = 1.0 / (inverse_min - u * (inverse_min - inverse_max))
    centers_x = rng.uniform(0, width, size=count)
    centers_y = rng.uniform(0, height, size=count)
    for diameter, cx, cy in zip(diameters, centers_x, centers_y):
        radius_px = 0.5 * diameter / resolution_m
        depth, rim = 0.2 * diameter, 0.04 * diameter
        reach = max(2, int(math.ceil(3.0 * radius_px)))
        x0, x1 = max(0, int(cx) - reach), min(width, int(cx) + reach + 1)
        y0, y1 = max(0, int(cy) - reach), min(height, int(cy) + reach + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1]
        r = np.hypot(xx - cx, yy - cy) / max(radius_px, 1e-6)
        profile = np.where(
            r < 1.0,
            -depth + (depth + rim) * r * r,
            rim / np.maximum(r, 1.0) ** 3,
        )
        surface[y0:y1, x0:x1] += profile


@dataclass(frozen=True)
class SyntheticDemSpec:
    size: int
    resolution_m: float
    latitude_deg: float = -85.0
    longitude_deg: float = 30.0
    sigma_m: float = 150.0
    hurst: float = 0.8
    craters: int = 40
    crater_min_m: float = 100.0
    crater_max_m: float = 3000.0
    tilt_m: float = 0.0
    seed: int = 1


def synthetic_dem(spec: SyntheticDemSpec) -> DemGrid:
    rng = np.random.default_rng(spec.seed)
    surface = fbm_surface(spec.size, spec.size, hurst=spec.hurst, sigma_m=spec.sigma_m,
                          rng=rng)
    if spec.craters:
        add_craters(surface, spec.resolution_m, spec.craters, min_diameter_m=spec.crater_min_m,
                    max_diameter_m=spec.crater_max_m, rng=rng)
    if spec.tilt_m:
        ramp = np.linspace(-0.5, 0.5, spec.size)
        surface += spec.tilt_m * ramp[None, :]
    projection = ProjectionParameters.south_polar(MOON_RADIUS_M)
    x, y = project_south_polar(math.radians(spec.latitude_deg),
                               math.radians(spec.longitude_deg), projection)
    half = spec.size * spec.resolution_m / 2.0
    transform = np.array(
        (x - half, spec.resolution_m, 0.0, y + half, 0.0, -spec.resolution_m),
        dtype=np.float64,
    )
    return DemGrid(np.ascontiguousarray(surface, dtype=np.float32), transform, projection)


def config1_dem() -> DemGrid:
    """512 x 512 at 20 m, fBm sigma 150 m, 40 craters 100-3000 m (seed 1)."""
    return synthetic_dem(SyntheticDemSpec(512, 20.0, seed=1))


def site_dem(size: int = 4096, resolution_m: float = 5.0, *, craters: int = 600,
             crater_max_m: float = 8000.0, seed: int = 2) -> DemGrid:
    """Site-scale primary DEM of the site configuration (4096 x 4096 at 5 m)."""
    return synthetic_dem(SyntheticDemSpec(size, resolution_m, craters=craters,
                                          crater_max_m=crater_max_m, seed=seed))


def regional_dem(size: int = 2000, resolution_m: float = 240.0, *, seed: int = 2) -> DemGrid:
    """Regional DEM: fBm sigma 1.2 km plus a 2 km planar tilt."""
    return synthetic_dem(SyntheticDemSpec(size, resolution_m, sigma_m=1200.0, craters=0,
                                          tilt_m=2000.0, seed=seed + 1000))


def multisite_specs(count: int = 64, *, seed: int = 64) -> list[SyntheticDemSpec]:
    """The uneven multi-site batch: sides log-uniform in [256, 2048] px,
    resolution from {5, 10, 20, 40} m, latitudes -83 to -89.5 deg, any
    longitude; crater sizes scale with the site extent."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        size = int(round(math.exp(rng.uniform(math.log(256), math.log(2048)))))
        resolution = float(rng.choice((5.0, 10.0, 20.0, 40.0)))
        extent = size * resolution
        specs.append(SyntheticDemSpec(
            size, resolution, latitude_deg=float(rng.uniform(-89.5, -83.0)),
            longitude_deg=float(rng.uniform(0.0, 360.0)),
            craters=max(8, size * size // 20000), crater_max_m=min(8000.0, extent / 4.0),
            seed=seed * 1000 + i))
    return specs


def polar_regional_dem(size: int = 2000, resolution_m: float = 240.0, *,
                       seed: int = 2) -> DemGrid:
    """Regional DEM centred on the pole (480 km across at the defaults), so
    that it surrounds every site of the multi-site batch."""
    return synthetic_dem(SyntheticDemSpec(size, resolution_m, latitude_deg=-90.0,
                                          longitude_deg=0.0, sigma_m=1200.0, craters=0,
                                          tilt_m=2000.0, seed=seed + 1000))


def hours_between(start: str, stop: str, step_hours: float) -> np.ndarray:
    """Elapsed hours of a regular time axis [start, stop] (inclusive)."""
    t0 = np.datetime64(start)
    t1 = np.datetime64(stop)
    total = (t1 - t0) / np.timedelta64(1, "h")
    count = int(math.floor(total / step_hours + 1e-9)) + 1
    return np.arange(count, dtype=np.float64) * step_hours


def sun_vectors(hours: np.ndarray, *, longitude0_deg: float = 0.0) -> np.ndarray:
    """Moon-ME Sun vectors (m) at 1 AU for elapsed hours."""
    days = np.asarray(hours, dtype=np.float64) / 24.0
    latitude = np.radians(1.54) * np.sin(2.0 * np.pi * days / 346.6)
    longitude = np.radians(longitude0_deg) - 2.0 * np.pi * days / 29.53
    cos_lat = np.cos(latitude)
    return np.ascontiguousarray(
        AU_M * np.stack((cos_lat * np.cos(longitude), cos_lat * np.sin(longitude),
                         np.sin(latitude)), axis=1))


def earth_vectors(hours: np.ndarray) -> np.ndarray:
    """Moon-ME Earth vectors (m) with optical librations."""
    days = np.asarray(hours, dtype=np.float64) / 24.0
    latitude = np.radians(6.7) * np.sin(2.0 * np.pi * days / 27.21)
    longitude = np.radians(7.9) * np.sin(2.0 * np.pi * days / 27.55)
    cos_lat = np.cos(latitude)
    return np.ascontiguousarray(
        EARTH_DISTANCE_M * np.stack((cos_lat * np.cos(longitude),
                                     cos_lat * np.sin(longitude), np.sin(latitude)), axis=1))


def config1_sun_vectors() -> np.ndarray:
    """2029-01-01 to 2029-02-01 at 6 h steps: 125 vectors."""
    return sun_vectors(hours_between("2029-01-01T00", "2029-02-01T00", 6.0))
