"""Host data contracts of the horizon path (mirrors
src/lunarscout/_numba_horizon/contract.py and geometry.py:25-115).

The session classes accept these types or the reference's own (they only read
attributes), so reference pipelines can hand their objects straight in.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

PATCH_SIZE = 128
AZIMUTH_COUNT = 1440
PIXEL_COUNT = PATCH_SIZE * PATCH_SIZE
SEGMENT_FIELD_COUNT = 18
SEGMENT_FIELDS = (
    "start_pixel_x", "start_pixel_y", "x0", "y0", "a1", "a2", "a3", "a4",
    "b1", "b2", "b3", "b4", "s_start_km", "s_end_km",
    "s_start_chord_km", "planar_to_chord_c1", "planar_to_chord_c2",
    "planar_to_chord_c3",
)
SUPPORTED_SUBPATCH_SIZES = frozenset((2, 4, 8, 16, 32, 64, 128))
SLOPE_SENTINEL = np.float32(-np.inf)
MOON_RADIUS_M = 1_737_400.0


class ContractValidationError(ValueError):
    """An array contract is violated (raised before any device work)."""


@dataclass(frozen=True, slots=True)
class ProjectionParameters:
    """Spherical stereographic projection (geometry.py:25-41)."""

    radius_m: float
    latitude_origin_rad: float
    longitude_origin_rad: float
    scale: float
    false_easting_m: float
    false_northing_m: float

    @classmethod
    def from_array(cls, values: npt.ArrayLike) -> "ProjectionParameters":
        array = np.asarray(values, dtype=np.float64)
        if array.shape != (6,) or not np.all(np.isfinite(array)):
            raise ContractValidationError("projection parameters must be six finite values")
        return cls(*(float(v) for v in array))

    @classmethod
    def south_polar(cls, radius_m: float = MOON_RADIUS_M) -> "ProjectionParameters":
        return cls(radius_m, -math.pi / 2.0, 0.0, 1.0, 0.0, 0.0)

    def as_array(self) -> np.ndarray:
        return np.array(
            (self.radius_m, self.latitude_origin_rad, self.longitude_origin_rad,
             self.scale, self.false_easting_m, self.false_northing_m),
            dtype=np.float64,
        )


def projection_array(projection) -> np.ndarray:
    return np.array(
        (projection.radius_m, projection.latitude_origin_rad,
         projection.longitude_origin_rad, projection.scale,
         projection.false_easting_m, projection.false_northing_m),
        dtype=np.float64,
    )


@dataclass(frozen=True, slots=True)
class DemGrid:
    """float32[y, x] elevations with a GDAL geotransform (geometry.py:44-115)."""

    elevation_m: npt.NDArray[np.float32]
    geo_transform: npt.NDArray[np.float64]
    projection: ProjectionParameters

    def __post_init__(self) -> None:
        e = self.elevation_m
        if (not isinstance(e, np.ndarray) or e.dtype != np.float32 or e.ndim != 2
                or not e.flags.c_contiguous):
            raise ContractValidationError("DEM elevation must be C-contiguous float32[y, x]")
        t = self.geo_transform
        if (not isinstance(t, np.ndarray) or t.dtype != np.float64 or t.shape != (6,)
                or not t.flags.c_contiguous or not np.all(np.isfinite(t))):
            raise ContractValidationError(
                "DEM geotransform must be six C-contiguous float64 values")
        if abs(t[1] * t[5] - t[2] * t[4]) < 1e-12:
            raise ContractValidationError("DEM geotransform is singular")

    @property
    def height(self) -> int:
        return self.elevation_m.shape[0]

    @property
    def width(self) -> int:
        return self.elevation_m.shape[1]

    @property
    def map_resolution_m(self) -> float:
        t = self.geo_transform
        return float((np.hypot(t[1], t[4]) + np.hypot(t[2], t[5])) * 0.5)


def map_parameters(dem) -> np.ndarray:
    """The 11 float32 map parameters of a DEM (pyramid.py:81-95)."""
    t = dem.geo_transform
    determinant = t[1] * t[5] - t[2] * t[4]
    p = dem.projection
    return np.array(
        (p.radius_m, p.scale, p.false_easting_m, p.false_northing_m, 1.0 / determinant, *t),
        dtype=np.float32,
    )


def projection_parameters(dem) -> np.ndarray:
    return projection_array(dem.projection).astype(np.float32)


@dataclass(frozen=True, slots=True)
class PyramidArrays:
    """Level 0, packed mips and the (level, offset, width, height) table."""

    level0: npt.NDArray[np.float32]
    mips: npt.NDArray[np.float32]
    levels: npt.NDArray[np.int32]
    map_parameters: npt.NDArray[np.float32]
    projection_parameters: npt.NDArray[np.float32]

    def __post_init__(self) -> None:
        if self.level0.dtype != np.float32 or self.level0.ndim != 2:
            raise ContractValidationError("pyramid level 0 must be float32[y, x]")
        if self.mips.dtype != np.float32 or self.mips.ndim != 1:
            raise ContractValidationError("pyramid mips must be float32[n]")
        if self.levels.dtype != np.int32 or self.levels.ndim != 2 or self.levels.shape[1] != 4:
            raise ContractValidationError("pyramid level metadata must be int32[L, 4]")
        expected = 0
        for index, (level, offset, width, height) in enumerate(self.levels):
            if level != index or width <= 0 or height <= 0:
                raise ContractValidationError("invalid pyramid level metadata")
            if index == 0:
                if offset != 0 or self.level0.shape != (height, width):
                    raise ContractValidationError("level-0 metadata does not match its array")
            else:
                if offset != expected:
                    raise ContractValidationError("pyramid mip offsets are not contiguous")
                expected += int(width) * int(height)
        if expected != self.mips.size:
            raise ContractValidationError("pyramid mip buffer length does not match metadata")


@dataclass(frozen=True, slots=True)
class ContractConfiguration:
    """Tile / azimuth / subpatch configuration (contract.py:110-153)."""

    tile_width: int
    tile_height: int
    azimuth_count: int
    subpatch_size: int
    dem_count: int
    primary_width: int
    primary_height: int

    def __post_init__(self) -> None:
        for name in ("tile_width", "tile_height", "azimuth_count", "dem_count",
                     "primary_width", "primary_height"):
            value = getattr(self, name)
            if not isinstance(value, int) or isinstance(value, bool) or value <= 0:
                raise ContractValidationError(f"{name} must be a positive integer")
        if self.subpatch_size not in SUPPORTED_SUBPATCH_SIZES:
            raise ContractValidationError(
                f"subpatch_size must be one of {sorted(SUPPORTED_SUBPATCH_SIZES)}")
        if 128 % self.subpatch_size:
            raise ContractValidationError("subpatch_size must evenly divide 128")
        if self.tile_width > 128 or self.tile_height > 128:
            raise ContractValidationError("tile dimensions cannot exceed 128 pixels")

    @property
    def pixel_count(self) -> int:
        return self.tile_width * self.tile_height

    @property
    def subpatches_per_dimension(self) -> int:
        return self.tile_width // self.subpatch_size + 2

    @property
    def subpatch_count(self) -> int:
        return self.subpatches_per_dimension ** 2

    @property
    def output_shape(self) -> tuple[int, int]:
        return self.pixel_count, self.azimuth_count


@dataclass(frozen=True, slots=True)
class SegmentTensor:
    """float32[A, C, D, 18] segments with their configuration."""

    values: npt.NDArray[np.float32]
    dem_ids: npt.NDArray[np.int32]
    configuration: ContractConfiguration

    def __post_init__(self) -> None:
        c = self.configuration
        expected = (c.azimuth_count, c.subpatch_count, c.dem_count, SEGMENT_FIELD_COUNT)
        if (self.values.dtype != np.float32 or self.values.shape != expected
                or not self.values.flags.c_contiguous):
            raise ContractValidationError(f"segment values must be float32{expected}")


@dataclass(frozen=True, slots=True)
class HorizonBuffers:
    """Pixel-major slopes float32[P, A] with -inf as the only sentinel."""

    slopes: npt.NDArray[np.float32]

    def __post_init__(self) -> None:
        if self.slopes.dtype != np.float32 or self.slopes.ndim != 2:
            raise ContractValidationError("slope buffer must be float32[P, A]")
        if np.any(np.isnan(self.slopes)) or np.any(np.isposinf(self.slopes)):
            raise ContractValidationError(
                "slope buffer may only use negative infinity as a sentinel")

    def degrees(self) -> npt.NDArray[np.float32]:
        """float32(arctan(slope) * float32(180)/float32(pi)), -inf preserved."""
        result = np.ascontiguousarray(
            np.arctan(self.slopes) * (np.float32(180.0) / np.float32(np.pi)),
            dtype=np.float32,
        )
        result[np.isneginf(self.slopes)] = SLOPE_SENTINEL
        return result

    def merge_pass(self, pass_slopes: npt.NDArray[np.float32]) -> "HorizonBuffers":
        if pass_slopes.shape != self.slopes.shape:
            raise ContractValidationError("DEM-pass slope buffer shape mismatch")
        return HorizonBuffers(np.ascontiguousarray(np.maximum(self.slopes, pass_slopes)))
