"""Drop-in ``LightmapCudaSession`` (src/lunarscout/_numba_horizon/lightmap_cuda.py:187-276).

Same constructor, ``iter_patch_tiles`` / ``iter_patch_fraction_tiles`` /
``iter_patch_margin_tiles`` signatures, lazily yielded per-time tiles and
error behaviour.  One device launch covers a large block of time steps (all
pixels x many times fill the GPU); host output stays bounded by that block.
"""

from __future__ import annotations

import ctypes
import hashlib
import threading
from collections.abc import Iterator

import numpy as np

from . import _native
from ._native import CudaBackendError, call, library, register
from .contract import AZIMUTH_COUNT, PATCH_SIZE, projection_array

SIGNAL_FRACTION = 0
SIGNAL_BYTES = 1
SIGNAL_MARGIN = 2
SIGNAL_PSR = 3
#: Time steps computed per device launch by the iterators.
DEVICE_TIME_BLOCK = 1024

__all__ = ["LightmapCudaSession", "CudaBackendError"]


def validate_vectors(vectors_m) -> np.ndarray:
    """float64 (time, 3), finite, non-empty (psr.py:17-26)."""
    values = np.ascontiguousarray(vectors_m, dtype=np.float64)
    if (values.ndim != 2 or values.shape[1:] != (3,) or values.shape[0] == 0
            or not np.all(np.isfinite(values))):
        raise ValueError("Moon-ME vectors must be finite values shaped (time, 3)")
    return values


def patch_elevations(dem, tile_y, tile_x, valid_height, valid_width) -> np.ndarray:
    patch = np.zeros((PATCH_SIZE, PATCH_SIZE), dtype=np.float32)
    patch[:valid_height, :valid_width] = dem.elevation_m[
        tile_y:tile_y + valid_height, tile_x:tile_x + valid_width]
    return patch


class DeviceVectors:
    """A float32 vector table resident on the device."""

    def __init__(self, context, vectors32: np.ndarray):
        self._context = context
        self.handle = ctypes.c_void_p()
        self.count = len(vectors32)
        call("ls200_vectors_create", context, np.ascontiguousarray(vectors32, np.float32),
             self.count, ctypes.byref(self.handle))

    def close(self, context_alive: bool = True) -> None:
        if self.handle and context_alive:
            library().ls200_vectors_destroy(self.handle)
        self.handle = ctypes.c_void_p()


class LightingContext:
    """Owns one ls200 context for a lighting session."""

    def __init__(self, device_id: int):
        handle = ctypes.c_void_p()
        lib = library()
        _native.check(lib.ls200_context_create(int(device_id), ctypes.byref(handle)),
                      "CUDA session")
        self.handle = handle
        self.lock = threading.Lock()
        self.vectors: DeviceVectors | None = None
        self.vector_key = None

    def resident_vectors(self, vectors32: np.ndarray, key) -> DeviceVectors:
        if self.vectors is None or self.vector_key != key:
            if self.vectors is not None:
                self.vectors.close()
            self.vectors = DeviceVectors(self.handle, vectors32)
            self.vector_key = key
        return self.vectors

    def close(self) -> None:
        if self.handle:
            if self.vectors is not None:
                self.vectors.close()
                self.vectors = None
            library().ls200_context_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class LightmapCudaSession:
    """Sun fraction / margin tiles of one horizon patch on the B200."""

    def __init__(self, *, device_id: int = 0, time_batch_size: int = 32) -> None:
        if time_batch_size < 1:
            raise ValueError("time_batch_size must be positive")
        self.time_batch_size = int(time_batch_size)
        self._context = LightingContext(device_id)
        self._lock = threading.Lock()

    def close(self) -> None:
        self._context.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _iter_patch_batches(self, dem, horizons_deg, body_vectors_m, *, tile_y: int,
                            tile_x: int, valid_height: int, valid_width: int, signal: str):
        vectors64 = validate_vectors(body_vectors_m)
        vectors = np.ascontiguousarray(vectors64, dtype=np.float32)
        horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
        if horizons.shape != (PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT):
            raise ValueError("horizons must have shape (128, 128, 1440)")
        if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
            raise ValueError("valid patch dimensions must be between 1 and 128")
        patch = patch_elevations(dem, tile_y, tile_x, valid_height, valid_width)
        geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
        projection = projection_array(dem.projection)
        key = hashlib.sha256(vectors.tobytes()).digest()
        code = {"fraction": SIGNAL_FRACTION, "margin": SIGNAL_MARGIN,
                "encoded": SIGNAL_BYTES}[signal]
        dtype = np.uint8 if code == SIGNAL_BYTES else np.float32
        total = len(vectors)
        block = max(self.time_batch_size, DEVICE_TIME_BLOCK)
        # Like the reference session, the lock is held for the whole patch
        # (across yields): the device tile buffers belong to one patch.
        with self._lock, self._context.lock:
            device_vectors = self._context.resident_vectors(vectors, key)
            call("ls200_lighting_load", self._context.handle, patch, geo, projection,
                 horizons.reshape(-1), int(tile_x), int(tile_y), int(valid_width),
                 int(valid_height))
            for block_start in range(0, total, block):
                count = min(block, total - block_start)
                out = np.empty((count, PATCH_SIZE, PATCH_SIZE), dtype=dtype)
                call("ls200_lighting_run", self._context.handle, device_vectors.handle,
                     block_start, count, code, out.ctypes.data)
                for start in range(0, count, self.time_batch_size):
                    stop = min(start + self.time_batch_size, count)
                    yield out[start:stop, :valid_height, :valid_width]

    def iter_patch_fraction_tiles(self, dem, horizons_deg, sun_vectors_m, *, tile_y: int,
                                  tile_x: int, valid_height: int = PATCH_SIZE,
                                  valid_width: int = PATCH_SIZE) -> Iterator[np.ndarray]:
        """float32 visible solar-disk fraction per time step."""
        for batch in self._iter_patch_batches(
                dem, horizons_deg, sun_vectors_m, tile_y=tile_y, tile_x=tile_x,
                valid_height=valid_height, valid_width=valid_width, signal="fraction"):
            for tile in batch:
                yield np.ascontiguousarray(tile)

    def iter_patch_margin_tiles(self, dem, horizons_deg, body_vectors_m, *, tile_y: int,
                                tile_x: int, valid_height: int = PATCH_SIZE,
                                valid_width: int = PATCH_SIZE) -> Iterator[np.ndarray]:
        """Body-centre elevation relative to the interpolated local horizon."""
        for batch in self._iter_patch_batches(
                dem, horizons_deg, body_vectors_m, tile_y=tile_y, tile_x=tile_x,
                valid_height=valid_height, valid_width=valid_width, signal="margin"):
            for tile in batch:
                yield np.ascontiguousarray(tile)

    def iter_patch_tiles(self, dem, horizons_deg, sun_vectors_m, *, tile_y: int, tile_x: int,
                         valid_height: int = PATCH_SIZE,
                         valid_width: int = PATCH_SIZE) -> Iterator[np.ndarray]:
        """uint8 lightmap bytes, int(float32(255) * fraction)."""
        for batch in self._iter_patch_batches(
                dem, horizons_deg, sun_vectors_m, tile_y=tile_y, tile_x=tile_x,
                valid_height=valid_height, valid_width=valid_width, signal="encoded"):
            for tile in batch:
                yield np.ascontiguousarray(tile)

    def mission_durations(self, dem, horizons_deg, sun_vectors_m, *, tile_y: int, tile_x: int,
                          valid_height: int, valid_width: int, sample_hours,
                          start_windows, earth_vectors_m=None, sun_threshold: float = 0.5,
                          earth_threshold: float = 0.0, days: bool = False) -> np.ndarray:
        """Longest right-censored condition run per candidate start window,
        float32 [I, valid_height, valid_width] (hours, or days): the condition
        (sun fraction >= sun_threshold [and Earth margin >= earth_threshold])
        evaluated and reduced on the device without materialising it
        (nh/mission_duration.py:164-256).  ``sample_hours`` f64[T] is the
        duration credited to each sample; ``start_windows`` int[I, 2] the
        (first, end) sample indices of each candidate start window."""
        import torch

        sun = np.ascontiguousarray(validate_vectors(sun_vectors_m), dtype=np.float32)
        earth = (None if earth_vectors_m is None else
                 np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32))
        if earth is not None and len(earth) != len(sun):
            raise ValueError("Earth and Sun vectors must share the time axis")
        hours = np.ascontiguousarray(sample_hours, dtype=np.float64)
        if hours.shape != (len(sun),):
            raise ValueError("sample_hours must have one entry per time step")
        windows = np.ascontiguousarray(start_windows, dtype=np.int32).reshape(-1, 2)
        horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
        if horizons.shape != (PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT):
            raise ValueError("horizons must have shape (128, 128, 1440)")
        if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
            raise ValueError("valid patch dimensions must be between 1 and 128")
        patch = torch.from_numpy(
            patch_elevations(dem, tile_y, tile_x, valid_height, valid_width)).cuda()
        device_horizons = torch.from_numpy(horizons).cuda()
        out = torch.empty((len(windows), PATCH_SIZE * PATCH_SIZE), dtype=torch.float32,
                          device="cuda")
        geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
        projection = projection_array(dem.projection)
        window = np.array([tile_x, tile_y, valid_width, valid_height], dtype=np.int32)
        torch.cuda.synchronize()
        with self._lock, self._context.lock:
            sun_table = DeviceVectors(self._context.handle, sun)
            earth_table = None if earth is None else DeviceVectors(self._context.handle, earth)
            try:
                call("ls200_mission_duration_device", self._context.handle, 1,
                     ctypes.c_void_p(patch.data_ptr()), geo.ctypes.data, projection.ctypes.data,
                     window.ctypes.data, ctypes.c_void_p(device_horizons.data_ptr()),
                     sun_table.handle, None if earth_table is None else earth_table.handle,
                     float(sun_threshold), float(earth_threshold), hours.ctypes.data,
                     windows.ctypes.data, len(windows), 1 if days else 0,
                     ctypes.c_void_p(out.data_ptr()))
            finally:
                sun_table.close()
                if earth_table is not None:
                    earth_table.close()
        grid = out.cpu().numpy().reshape(len(windows), PATCH_SIZE, PATCH_SIZE)
        return np.ascontiguousarray(grid[:, :valid_height, :valid_width])

    def safe_haven_durations(self, dem, horizons_deg, sun_vectors_m, earth_vectors_m, *,
                             tile_y: int, tile_x: int, valid_height: int, valid_width: int,
                             month_index_of, band_count: int, time_step_hours: float,
                             sunlight_threshold: float = 0.2,
                             earth_threshold_deg: float = 2.0) -> tuple[np.ndarray, ...]:
        """Per month band, the longest low-Sun run (fraction <
        ``sunlight_threshold``) that overlapped an Earth outage (margin <
        ``earth_threshold_deg``) in that band, times ``time_step_hours``:
        float32 ``[valid_height, valid_width]`` per band, NaN where the band
        saw no outage or only outages (reduce_safe_haven_patch_stream,
        safe_haven.py:75-243, over the streams of safe_haven_pipeline.py:240-272,
        evaluated and reduced on the device).  ``month_index_of`` int32[T]
        gives each time step's band (-1 for none)."""
        import torch

        sun = np.ascontiguousarray(validate_vectors(sun_vectors_m), dtype=np.float32)
        earth = np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32)
        if len(earth) != len(sun):
            raise ValueError("timestamps, Sun vectors, and Earth vectors must align")
        if not 0.0 <= sunlight_threshold <= 1.0:
            raise ValueError("sunlight_threshold must be between zero and one")
        if not np.isfinite(earth_threshold_deg):
            raise ValueError("earth_threshold_deg must be finite")
        if not np.isfinite(time_step_hours) or time_step_hours <= 0.0:
            raise ValueError("time_step_hours must be positive and finite")
        if isinstance(band_count, bool) or not isinstance(band_count, (int, np.integer)) \
                or band_count < 1:
            raise ValueError("band_count must be a positive integer")
        months = np.ascontiguousarray(month_index_of, dtype=np.int32)
        if months.shape != (len(sun),):
            raise ValueError("month_index_of must have shape (time_count,)")
        if np.any((months < -1) | (months >= band_count)):
            raise ValueError("month indices must be -1 or a band index")
        horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
        if horizons.shape != (PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT):
            raise ValueError("horizons must have shape (128, 128, 1440)")
        if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
            raise ValueError("valid patch dimensions must be between 1 and 128")
        patch = torch.from_numpy(
            patch_elevations(dem, tile_y, tile_x, valid_height, valid_width)).cuda()
        device_horizons = torch.from_numpy(horizons).cuda()
        out = torch.empty((int(band_count), PATCH_SIZE * PATCH_SIZE), dtype=torch.float32,
                          device="cuda")
        geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
        projection = projection_array(dem.projection)
        window = np.array([tile_x, tile_y, valid_width, valid_height], dtype=np.int32)
        torch.cuda.synchronize()
        with self._lock, self._context.lock:
            sun_table = DeviceVectors(self._context.handle, sun)
            earth_table = DeviceVectors(self._context.handle, earth)
            try:
                call("ls200_safe_haven_device", self._context.handle, 1,
                     ctypes.c_void_p(patch.data_ptr()), geo.ctypes.data, projection.ctypes.data,
                     window.ctypes.data, ctypes.c_void_p(device_horizons.data_ptr()),
                     sun_table.handle, earth_table.handle, float(sunlight_threshold),
                     float(earth_threshold_deg), float(np.float32(time_step_hours)),
                     months.ctypes.data, int(band_count), ctypes.c_void_p(out.data_ptr()))
            finally:
                sun_table.close()
                earth_table.close()
        grid = out.cpu().numpy().reshape(int(band_count), PATCH_SIZE, PATCH_SIZE)
        return tuple(np.ascontiguousarray(band[:valid_height, :valid_width]) for band in grid)

    def earth_visibility_fraction(self, dem, horizons_deg, earth_vectors_m, *, tile_y: int,
                                  tile_x: int, valid_height: int, valid_width: int,
                                  threshold_deg: float = 0.0) -> np.ndarray:
        """Share of the time steps at which the Earth's centre stands at least
        ``threshold_deg`` above the terrain horizon: the mean over time of
        (margin >= threshold) for the margins ``iter_patch_margin_tiles``
        yields (lightmap_cuda.py:125-145), float32 [valid_height,
        valid_width], counted on the device without materialising the
        margins."""
        import torch

        earth = np.ascontiguousarray(validate_vectors(earth_vectors_m), dtype=np.float32)
        if not np.isfinite(threshold_deg):
            raise ValueError("threshold_deg must be finite")
        horizons = np.ascontiguousarray(horizons_deg, dtype=np.float32)
        if horizons.shape != (PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT):
            raise ValueError("horizons must have shape (128, 128, 1440)")
        if not 1 <= valid_width <= PATCH_SIZE or not 1 <= valid_height <= PATCH_SIZE:
            raise ValueError("valid patch dimensions must be between 1 and 128")
        patch = torch.from_numpy(
            patch_elevations(dem, tile_y, tile_x, valid_height, valid_width)).cuda()
        device_horizons = torch.from_numpy(horizons).cuda()
        out = torch.empty(PATCH_SIZE * PATCH_SIZE, dtype=torch.float32, device="cuda")
        geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
        projection = projection_array(dem.projection)
        window = np.array([tile_x, tile_y, valid_width, valid_height], dtype=np.int32)
        torch.cuda.synchronize()
        with self._lock, self._context.lock:
            table = DeviceVectors(self._context.handle, earth)
            try:
                call("ls200_earth_visibility_device", self._context.handle, 1,
                     ctypes.c_void_p(patch.data_ptr()), geo.ctypes.data, projection.ctypes.data,
                     window.ctypes.data, ctypes.c_void_p(device_horizons.data_ptr()),
                     table.handle, float(threshold_deg), ctypes.c_void_p(out.data_ptr()))
            finally:
                table.close()
        grid = out.cpu().numpy().reshape(PATCH_SIZE, PATCH_SIZE)
        return np.ascontiguousarray(grid[:valid_height, :valid_width])

    def sun_fraction(self, horizons: np.ndarray, azimuth_deg, elevation_deg) -> np.ndarray:
        """Diagnostic: fraction of the disk at (azimuth, elevation) above each
        horizon row (lightmap.py:32-73)."""
        horizons = np.ascontiguousarray(horizons, dtype=np.float32).reshape(-1, AZIMUTH_COUNT)
        az = np.ascontiguousarray(np.broadcast_to(azimuth_deg, (len(horizons),)), np.float32)
        el = np.ascontiguousarray(np.broadcast_to(elevation_deg, (len(horizons),)), np.float32)
        out = np.empty(len(horizons), dtype=np.float32)
        with self._context.lock:
            call("ls200_sun_fraction", self._context.handle, horizons.reshape(-1), az, el,
                 len(horizons), out)
        return out
