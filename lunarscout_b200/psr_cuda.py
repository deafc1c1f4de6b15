"""Drop-in ``PsrCudaSession`` (src/lunarscout/_numba_horizon/psr_cuda.py:23-375).

Same constructor, ``allocate_pinned_horizon_buffer``, ``compute_patch``
signature, validation, resident-vector reuse and optional per-patch timing
callback; the kernel is the sm_100a PSR kernel of ``libls200.so``.
"""

from __future__ import annotations

import ctypes
import threading
import time
from collections.abc import Callable
from dataclasses import dataclass

import numpy as np

from ._native import CudaBackendError, call, pinned_empty
from .contract import AZIMUTH_COUNT, PATCH_SIZE, projection_array
from .lightmap_cuda import LightingContext, patch_elevations

__all__ = ["PsrCudaSession", "PsrCudaPatchTimings", "CudaBackendError",
           "reduce_sun_vectors_for_psr"]

#: Viewpoints x azimuth bins of the reduction: the most vectors it keeps.
MAX_REDUCED_VECTORS = 5 * AZIMUTH_COUNT


def _validate_moon_vectors(vectors_m) -> np.ndarray:
    values = np.ascontiguousarray(vectors_m, dtype=np.float64)
    if (values.ndim != 2 or values.shape[1:] != (3,) or values.shape[0] == 0
            or not np.all(np.isfinite(values))):
        raise ValueError("Moon-ME vectors must be finite values shaped (time, 3)")
    return values


def reduce_vectors_on(context_handle, dem, sun_vectors_m) -> tuple[np.ndarray, np.ndarray]:
    """The PSR vector reduction on an existing ls200 context (see
    reduce_sun_vectors_for_psr)."""
    vectors = _validate_moon_vectors(sun_vectors_m)
    elevation = np.ascontiguousarray(dem.elevation_m, dtype=np.float32)
    height, width = elevation.shape
    indices = np.empty(MAX_REDUCED_VECTORS, dtype=np.int64)
    kept = ctypes.c_int(0)
    call("ls200_psr_reduce_vectors", context_handle, elevation, int(width), int(height),
         np.ascontiguousarray(dem.geo_transform, dtype=np.float64),
         projection_array(dem.projection), vectors, len(vectors), indices.ctypes.data,
         ctypes.byref(kept))
    indices = np.ascontiguousarray(indices[:kept.value])
    return np.ascontiguousarray(vectors[indices]), indices


def reduce_sun_vectors_for_psr(dem, sun_vectors_m, *,
                               device_id: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Drop-in for reduce_sun_vectors_for_psr (src/lunarscout/_numba_horizon/
    psr.py:61-91), computed on the device: per viewpoint (the DEM's four
    corner pixels and its centre pixel) and 0.25-deg azimuth bin the vector
    with the highest elevation (first on ties), deduplicated in order of first
    appearance.  Returns (float64 reduced vectors, int64 indices)."""
    context = LightingContext(device_id)
    try:
        return reduce_vectors_on(context.handle, dem, sun_vectors_m)
    finally:
        context.close()


@dataclass(frozen=True, slots=True)
class PsrCudaPatchTimings:
    """Boundary timings of one PSR patch (psr_cuda.py:23-43)."""

    tile_y: int
    tile_x: int
    host_preparation_seconds: float
    h2d_dem_seconds: float
    h2d_metadata_seconds: float
    h2d_horizon_seconds: float
    h2d_vectors_seconds: float
    kernel_launch_seconds: float
    kernel_execution_seconds: float
    synchronization_boundary_seconds: float
    d2h_result_seconds: float
    total_seconds: float


class PsrCudaSession:
    """Permanently-shadowed-region masks of horizon patches on the B200."""

    def __init__(self, device_id: int = 0, *,
                 timing_callback: Callable[[PsrCudaPatchTimings], None] | None = None) -> None:
        self._context = LightingContext(device_id)
        self._lock = threading.Lock()
        self._timing_callback = timing_callback
        self._resident: np.ndarray | None = None

    def close(self) -> None:
        self._context.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def reduce_sun_vectors(self, dem, sun_vectors_m) -> tuple[np.ndarray, np.ndarray]:
        """reduce_sun_vectors_for_psr on this session's device."""
        with self._lock, self._context.lock:
            return reduce_vectors_on(self._context.handle, dem, sun_vectors_m)

    def allocate_pinned_horizon_buffer(self) -> np.ndarray:
        """Page-locked float32 (128, 128, 1440) buffer for direct decode + H2D."""
        return pinned_empty((PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT), np.float32)

    def compute_patch(self, dem, horizons_deg, sun_vectors_m, *, tile_y: int, tile_x: int,
                      valid_height: int = PATCH_SIZE,
                      valid_width: int = PATCH_SIZE) -> np.ndarray:
        total_started = time.perf_counter()
        if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
            raise ValueError("valid patch dimensions must be between 1 and 128")
        if (tile_x < 0 or tile_y < 0 or tile_x + valid_width > dem.width
                or tile_y + valid_height > dem.height):
            raise ValueError("PSR patch falls outside the DEM")
        horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
        if horizons.shape != (PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT):
            raise ValueError("horizons must have shape (128, 128, 1440)")
        if not np.all(np.isfinite(horizons)):
            raise ValueError("horizons must contain finite elevations")
        vectors = np.ascontiguousarray(sun_vectors_m, dtype=np.float32)
        if (vectors.ndim != 2 or vectors.shape[1:] != (3,) or vectors.shape[0] == 0
                or not np.all(np.isfinite(vectors))):
            raise ValueError("Sun vectors must be finite values shaped (time, 3)")
        patch = patch_elevations(dem, tile_y, tile_x, valid_height, valid_width)
        geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
        projection = projection_array(dem.projection)
        host_seconds = time.perf_counter() - total_started
        output = np.empty((PATCH_SIZE, PATCH_SIZE), dtype=np.uint8)
        with self._lock, self._context.lock:
            started = time.perf_counter()
            key = (vectors.shape, vectors.tobytes())
            reused = self._resident is not None and self._context.vector_key == key
            device_vectors = self._context.resident_vectors(vectors, key)
            vectors_seconds = 0.0 if reused else time.perf_counter() - started
            started = time.perf_counter()
            call("ls200_lighting_load", self._context.handle, patch, geo, projection,
                 horizons.reshape(-1), int(tile_x), int(tile_y), int(valid_width),
                 int(valid_height))
            load_seconds = time.perf_counter() - started
            started = time.perf_counter()
            call("ls200_psr_run", self._context.handle, device_vectors.handle,
                 output.ctypes.data)
            run_seconds = time.perf_counter() - started
            self._resident = vectors
        result = np.ascontiguousarray(output[:valid_height, :valid_width])
        if self._timing_callback is not None:
            self._timing_callback(PsrCudaPatchTimings(
                tile_y=tile_y, tile_x=tile_x, host_preparation_seconds=host_seconds,
                h2d_dem_seconds=0.0, h2d_metadata_seconds=0.0, h2d_horizon_seconds=load_seconds,
                h2d_vectors_seconds=vectors_seconds, kernel_launch_seconds=0.0,
                kernel_execution_seconds=run_seconds, synchronization_boundary_seconds=run_seconds,
                d2h_result_seconds=0.0, total_seconds=time.perf_counter() - total_started))
        return result
