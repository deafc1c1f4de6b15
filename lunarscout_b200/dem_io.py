"""DEM files and the sibling ``.pyr.bin`` maximum-pyramid cache.

DEM container: the reference reads stereographic GeoTIFFs through rasterio
(ls/products.py:97-175); rasterio and pyproj are not part of this runtime, so
a DEM travels as an ``.npz`` holding ``elevation_m`` float32[y, x],
``geo_transform`` float64[6] (GDAL order) and ``projection`` float64[6]
(radius m, latitude / longitude origin rad, scale, false easting / northing m)
— exactly the DemGrid the reference builds from the GeoTIFF.

Pyramid cache (nh/pyramid.py:34-75): a headerless little-endian float32 mip
payload beside the DEM (``dem.pyr.bin``), validated only by its length, and
atomically replaced when it is rebuilt.
"""

from __future__ import annotations

import os
import uuid
from pathlib import Path

import numpy as np

from .contract import (
    DemGrid,
    ProjectionParameters,
    PyramidArrays,
    map_parameters,
    projection_parameters,
)


class DemFormatError(ValueError):
    """The file is not a DEM container this runtime reads."""


def save_dem(path, dem: DemGrid) -> Path:
    target = Path(path)
    if target.suffix.lower() != ".npz":
        raise DemFormatError("DEM containers use the .npz extension")
    target.parent.mkdir(parents=True, exist_ok=True)
    with target.open("wb") as handle:
        np.savez(handle, elevation_m=dem.elevation_m, geo_transform=dem.geo_transform,
                 projection=dem.projection.as_array())
    return target


def load_dem(path) -> DemGrid:
    source = Path(path)
    if source.suffix.lower() != ".npz":
        raise DemFormatError(
            f"unsupported DEM file {source.name}: expected an .npz DEM container")
    try:
        with np.load(source, allow_pickle=False) as data:
            elevation = np.ascontiguousarray(data["elevation_m"], dtype=np.float32)
            transform = np.ascontiguousarray(data["geo_transform"], dtype=np.float64)
            projection = ProjectionParameters.from_array(data["projection"])
    except (KeyError, OSError, ValueError) as error:
        raise DemFormatError(f"{source.name} is not a readable DEM container: {error}") from error
    return DemGrid(elevation, transform, projection)


def pyramid_layout(width: int, height: int) -> tuple[np.ndarray, int]:
    """(level, offset, width, height) rows of the factor-four max pyramid down
    to 1x1, and the packed mip element count (nh/pyramid.py:19-31)."""
    shapes = [(int(height), int(width))]
    while shapes[-1] != (1, 1):
        h, w = shapes[-1]
        shapes.append(((h + 3) // 4, (w + 3) // 4))
    levels = np.empty((len(shapes), 4), dtype=np.int32)
    offset = 0
    for level, (h, w) in enumerate(shapes):
        levels[level] = (level, 0 if level == 0 else offset, w, h)
        if level > 0:
            offset += w * h
    return levels, offset


def pyramid_cache_path(dem_path) -> Path:
    return Path(dem_path).with_suffix(".pyr.bin")


def load_max_pyramid_cache(dem: DemGrid, path) -> PyramidArrays:
    """Raises OSError / ValueError when the cache is missing or the wrong length."""
    levels, expected = pyramid_layout(dem.width, dem.height)
    mips = np.fromfile(Path(path), dtype="<f4")
    if mips.size != expected:
        raise ValueError(f"pyramid cache has {mips.size} float32 values; expected {expected}")
    return PyramidArrays(dem.elevation_m, np.ascontiguousarray(mips, dtype=np.float32), levels,
                         map_parameters(dem), projection_parameters(dem))


def write_max_pyramid_cache(pyramid: PyramidArrays, path) -> Path:
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    staging = target.with_name(f".{target.name}.{uuid.uuid4().hex}.tmp")
    try:
        with staging.open("wb") as handle:
            np.asarray(pyramid.mips, dtype="<f4").tofile(handle)
            handle.flush()
            os.fsync(handle.fileno())
        os.replace(staging, target)
    except BaseException:
        try:
            staging.unlink(missing_ok=True)
        except OSError:
            pass
        raise
    return target
