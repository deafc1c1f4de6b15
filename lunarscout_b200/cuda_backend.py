"""Drop-in ``CudaSession`` for the horizon march on B200.

Mirrors src/lunarscout/_numba_horizon/cuda_backend.py:1143-1577: the same
constructor, ``info``, ``build_max_pyramid``, ``subpatch_hierarchical_pass``
and ``subpatch_hierarchical_all_passes`` signatures, return types and error
behaviour, backed by the sm_100a kernels of ``libls200.so``.

Constructing a session is the explicit boundary that touches CUDA; importing
this module does not.
"""

from __future__ import annotations

import ctypes
import threading
import time
import weakref
from dataclasses import dataclass

import numpy as np

from . import _native
from ._native import CudaBackendError, CudaExecutionError, call, library
from .contract import PyramidArrays, map_parameters, projection_parameters

__all__ = ["CudaBackendError", "CudaExecutionError", "CudaDeviceInfo", "CudaSession",
           "DeviceDem", "SiteTile", "BatchConfig", "TRAVERSALS"]

#: Traversals of the batched march: the reference's ("exact", bit-identical to
#: the drop-in), the skip ladder, and both in the relative FP32 arithmetic
#: (coordinates and heights relative to a local origin; within ~1e-4 deg of
#: the FP64 restatement of the march, not bit-identical to the reference).
TRAVERSALS = {"exact": 0, "ladder": 1, "relative": 2, "relative-ladder": 3}

# Slope arrays returned by the march calls live in recycled pinned memory
# (fresh, ordinary numpy arrays to the caller).
_OUTPUTS = _native.PinnedPool(keep=2)


@dataclass(frozen=True, slots=True)
class CudaDeviceInfo:
    name: str
    compute_capability: tuple[int, int]


@dataclass(frozen=True, slots=True)
class SiteTile:
    """One 128x128 tile of one site for :meth:`CudaSession.march_sites`."""

    dems: tuple  # DeviceDem, pass order, primary first
    tile_column: int
    tile_row: int
    maximum_distance_m: float = 1_000_000.0
    observer_elevation_m: float = 0.0


@dataclass(frozen=True, slots=True)
class BatchConfig:
    """Launch configuration of the persistent multi-site march:
    ``lanes_per_azimuth`` adjacent pixels of one azimuth per 32-ray warp job
    (a power of two up to 32; the job spans 32/lanes azimuths) and ``min_blocks``
    resident 128-thread blocks per SM (8 at 64 registers or 6 at 80)."""

    lanes_per_azimuth: int = 2
    min_blocks: int = 8


class _SiteTileStruct(ctypes.Structure):
    """ls200_site_tile (include/ls200.h)."""

    _fields_ = [("dems", ctypes.c_void_p), ("dem_count", ctypes.c_int),
                ("tile_column", ctypes.c_int), ("tile_row", ctypes.c_int),
                ("maximum_distance_m", ctypes.c_double),
                ("observer_elevation_m", ctypes.c_float)]


def site_tile_structs(tiles):
    """ls200_site_tile array for ``tiles`` (SiteTile) and the handle arrays it
    points into (keep both alive for the call)."""
    tiles = list(tiles)
    if not tiles:
        raise ValueError("at least one tile is required")
    handle_arrays = []
    structs = (_SiteTileStruct * len(tiles))()
    for slot, tile in zip(structs, tiles):
        handles = (ctypes.c_void_p * len(tile.dems))(*[d.handle.value for d in tile.dems])
        handle_arrays.append(handles)
        slot.dems = ctypes.cast(handles, ctypes.c_void_p)
        slot.dem_count = len(tile.dems)
        slot.tile_column = int(tile.tile_column)
        slot.tile_row = int(tile.tile_row)
        slot.maximum_distance_m = float(tile.maximum_distance_m)
        slot.observer_elevation_m = float(tile.observer_elevation_m)
    return structs, handle_arrays


class DeviceDem:
    """A DEM (level 0 + max pyramid + georeference) resident on the device."""

    def __init__(self, session: "CudaSession", handle: int, width: int, height: int):
        self._session = session
        self.handle = ctypes.c_void_p(handle)
        self.width = width
        self.height = height

    def close(self) -> None:
        # The context releases its DEMs itself; only an open session frees one.
        if self.handle and self._session._ctx:
            library().ls200_dem_destroy(self.handle)
        self.handle = ctypes.c_void_p(None)

    def __del__(self):  # pragma: no cover - best effort release
        try:
            self.close()
        except Exception:
            pass


def _pyramid_geo(pyramid) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(geo_transform f64[6], projection f64[6], map_parameters f32[11])."""
    mp = np.ascontiguousarray(pyramid.map_parameters, dtype=np.float32)
    pp = np.ascontiguousarray(pyramid.projection_parameters, dtype=np.float64)
    return np.ascontiguousarray(mp[5:11], dtype=np.float64), pp, mp


class CudaSession:
    """An explicitly initialised B200 session (one device, one stream)."""

    def __init__(self, device_id: int = 0, *, production_concurrency: int = 1) -> None:
        if production_concurrency < 1:
            raise ValueError("production_concurrency must be positive")
        self._production_concurrency = production_concurrency
        handle = ctypes.c_void_p()
        try:
            lib = library()
        except CudaBackendError:
            raise
        _native.check(lib.ls200_context_create(int(device_id), ctypes.byref(handle)),
                      "CUDA session")
        self._ctx = handle
        self.device_id = int(device_id)
        name = ctypes.create_string_buffer(256)
        major, minor, sms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("ls200_device_info", self._ctx, name, 256, ctypes.byref(major),
             ctypes.byref(minor), ctypes.byref(sms))
        self.info = CudaDeviceInfo(name.value.decode(), (major.value, minor.value))
        self.sm_count = sms.value
        self._lock = threading.Lock()
        self._dems = weakref.WeakSet()
        self._production_pyramids = None
        self._production_device_dems = None
        self._production_timings = threading.local()

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            for dem in list(self._dems):
                dem.close()
            library().ls200_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def context(self) -> ctypes.c_void_p:
        return self._ctx

    @property
    def last_production_timings(self):
        return getattr(self._production_timings, "value", None)

    def set_stream(self, stream_handle: int | None) -> None:
        """Run later work on an external cudaStream_t (e.g. torch's; 0 is the
        legacy default stream); None goes back to the session's own stream."""
        if stream_handle is None:
            call("ls200_reset_stream", self._ctx)
        else:
            call("ls200_set_stream", self._ctx, ctypes.c_void_p(stream_handle))

    def synchronize(self) -> None:
        call("ls200_synchronize", self._ctx)

    # -- DEMs and pyramids --------------------------------------------------
    def upload_dem(self, level0: np.ndarray, geo_transform, projection, map_params=None,
                   mips: np.ndarray | None = None) -> DeviceDem:
        """Upload a DEM; builds its max pyramid on the device unless given."""
        level0 = np.ascontiguousarray(level0, dtype=np.float32)
        height, width = level0.shape
        geo = np.ascontiguousarray(geo_transform, dtype=np.float64)
        proj = np.ascontiguousarray(projection, dtype=np.float64)
        if map_params is None:
            determinant = geo[1] * geo[5] - geo[2] * geo[4]
            map_params = np.array(
                (proj[0], proj[3], proj[4], proj[5], 1.0 / determinant, *geo), dtype=np.float32)
        mp = np.ascontiguousarray(map_params, dtype=np.float32)
        handle = ctypes.c_void_p()
        mips_ptr = None
        if mips is not None:
            mips = np.ascontiguousarray(mips, dtype=np.float32)
            mips_ptr = mips.ctypes.data
        call("ls200_dem_create", self._ctx, level0, width, height, mips_ptr, geo, proj, mp,
             ctypes.byref(handle))
        dem = DeviceDem(self, handle.value, width, height)
        self._dems.add(dem)
        return dem

    def upload_pyramid(self, pyramid, dem=None) -> DeviceDem:
        """Upload a PyramidArrays (level 0 + mips).  A pyramid carries its
        georeference only as float32 map and projection parameters, which is
        enough for the march; segment fitting needs the float64
        geotransform and projection, so callers that fit segments on the
        device pass the DemGrid the pyramid was built from (float32 rounds
        the polar latitude origin past -pi/2 and moves the observers)."""
        geo, proj, mp = _pyramid_geo(pyramid)
        if dem is not None:
            from .contract import projection_array

            geo = np.ascontiguousarray(dem.geo_transform, dtype=np.float64)
            proj = projection_array(dem.projection)
        mips = np.ascontiguousarray(pyramid.mips, dtype=np.float32)
        return self.upload_dem(pyramid.level0, geo, proj, mp, mips if mips.size else None)

    def upload_dem_grid(self, dem) -> DeviceDem:
        from .contract import projection_array

        return self.upload_dem(dem.elevation_m, dem.geo_transform,
                               projection_array(dem.projection), map_parameters(dem))

    @staticmethod
    def pyramid_layout(width: int, height: int) -> tuple[np.ndarray, int]:
        count, mip_count = ctypes.c_int(), ctypes.c_int64()
        levels = np.zeros((32, 4), dtype=np.int32)
        call("ls200_pyramid_layout", int(width), int(height), levels.ctypes.data, 32,
             ctypes.byref(count), ctypes.byref(mip_count))
        return levels[: count.value].copy(), int(mip_count.value)

    def build_max_pyramid(self, dem) -> PyramidArrays:
        """Production factor-four max pyramid built on the device
        (cuda_backend.py:1260-1281)."""
        level0 = np.ascontiguousarray(dem.elevation_m, dtype=np.float32)
        levels, mip_count = self.pyramid_layout(level0.shape[1], level0.shape[0])
        mips = np.empty(max(mip_count, 1), dtype=np.float32)
        call("ls200_build_max_pyramid", self._ctx, level0, level0.shape[1], level0.shape[0],
             mips)
        return PyramidArrays(level0, mips[:mip_count].copy(), levels, map_parameters(dem),
                             projection_parameters(dem))

    def _prepare_production_pyramids(self, pyramids) -> list[DeviceDem]:
        """Keep immutable pyramids resident across patches, keyed by identity
        (cuda_backend.py:1231-1258)."""
        host = tuple(pyramids)
        with self._lock:
            cached = self._production_pyramids
            if (cached is not None and len(host) == len(cached)
                    and all(a is b for a, b in zip(host, cached))):
                return self._production_device_dems
            if self._production_device_dems:
                for dem in self._production_device_dems:
                    dem.close()
            device = [self.upload_pyramid(p) for p in host]
            self._production_pyramids = host
            self._production_device_dems = device
            return device

    # -- the march ---------------------------------------------------------
    @staticmethod
    def _segments(segment_values, tile_width, subpatch_size):
        segments = np.ascontiguousarray(segment_values, dtype=np.float32)
        if segments.ndim != 4 or segments.shape[-1] != 18:
            raise ValueError("segment_values must have shape (azimuth, center, DEM, 18)")
        expected_centers = (tile_width // subpatch_size + 2) ** 2
        if segments.shape[1] != expected_centers:
            raise ValueError("segment center count does not match tile/subpatch layout")
        return segments

    def subpatch_hierarchical_pass(
        self, segment_values, primary_pyramid, active_pyramid, *, tile_column: int,
        tile_row: int, tile_width: int, tile_height: int, subpatch_size: int,
        pass_index: int, observer_elevation_m: float = 0.0, slopes=None,
    ) -> np.ndarray:
        """One production DEM pass in slope units (cuda_backend.py:1390-1443)."""
        segments = self._segments(segment_values, tile_width, subpatch_size)
        if not 0 <= pass_index < segments.shape[2]:
            raise ValueError("pass_index is outside the segment DEM axis")
        output_shape = (tile_width * tile_height, segments.shape[0])
        slopes_in = None
        if slopes is not None:
            slopes_in = np.ascontiguousarray(slopes, dtype=np.float32)
            if slopes_in.shape != output_shape:
                raise ValueError(f"slopes must have shape {output_shape}")
        primary = self.upload_pyramid(primary_pyramid)
        active = primary if active_pyramid is primary_pyramid else self.upload_pyramid(
            active_pyramid)
        out = _OUTPUTS.empty(output_shape, np.float32)
        try:
            call("ls200_march_pass", self._ctx, segments, segments.shape[0], segments.shape[1],
                 segments.shape[2], primary.handle, active.handle, int(tile_column),
                 int(tile_row), int(tile_width), int(tile_height), int(subpatch_size),
                 int(pass_index), float(observer_elevation_m),
                 None if slopes_in is None else slopes_in.ctypes.data, out)
        finally:
            if active is not primary:
                active.close()
            primary.close()
        return out

    def subpatch_hierarchical_all_passes(
        self, segment_values, pyramids, *, tile_column: int, tile_row: int,
        tile_width: int, tile_height: int, subpatch_size: int,
        observer_elevation_m: float = 0.0,
    ) -> tuple[np.ndarray, list[float]]:
        """Every DEM pass on one resident slope buffer; returns (slopes
        float32[P, A], per-pass CUDA-event seconds) (cuda_backend.py:1445-1552)."""
        segments = self._segments(segment_values, tile_width, subpatch_size)
        if len(pyramids) != segments.shape[2]:
            raise ValueError("pyramid count must match the segment DEM axis")
        dems = self._prepare_production_pyramids(pyramids)
        handles = (ctypes.c_void_p * len(dems))(*[d.handle.value for d in dems])
        out = _OUTPUTS.empty((tile_width * tile_height, segments.shape[0]), np.float32)
        seconds = np.zeros(len(dems), dtype=np.float64)
        started = time.perf_counter()
        call("ls200_march_all_passes", self._ctx, segments, segments.shape[0],
             segments.shape[1], segments.shape[2], handles, int(tile_column), int(tile_row),
             int(tile_width), int(tile_height), int(subpatch_size),
             float(observer_elevation_m), out, seconds.ctypes.data)
        self._production_timings.value = {
            "boundary_wall_seconds": time.perf_counter() - started,
            "kernel_seconds": float(seconds.sum()),
        }
        return out, [float(s) for s in seconds]

    # -- segment generation and diagnostics --------------------------------
    def generate_segments(self, dems, *, tile_column: int, tile_row: int,
                          tile_width: int = 128, azimuth_count: int = 1440,
                          maximum_distance_m: float = 1_000_000.0,
                          observer_elevation_m: float = 0.0,
                          subpatch_size: int = 8) -> np.ndarray:
        """Segment tensor float32[A, C, D, 18] computed on the device
        (geometry.py:575-673).  ``dems`` are DeviceDem handles."""
        handles = (ctypes.c_void_p * len(dems))(*[d.handle.value for d in dems])
        count = tile_width // subpatch_size + 2
        out = np.empty((azimuth_count, count * count, len(dems), 18), dtype=np.float32)
        call("ls200_segments", self._ctx, handles, len(dems), int(tile_column), int(tile_row),
             int(tile_width), int(azimuth_count), float(maximum_distance_m),
             float(observer_elevation_m), int(subpatch_size), out)
        return out

    def set_counting(self, enabled: bool) -> None:
        call("ls200_set_counting", self._ctx, 1 if enabled else 0)

    def last_counters(self) -> tuple[int, int, int]:
        """(node visits, level-0 samples, ray steps) of the last counted march."""
        visits, samples, steps = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        call("ls200_last_counters", self._ctx, ctypes.byref(visits), ctypes.byref(samples),
             ctypes.byref(steps))
        return int(visits.value), int(samples.value), int(steps.value)

    def march_all_passes_device(self, device_segments: int, azimuth_count: int,
                                center_count: int, dems, *, tile_column: int, tile_row: int,
                                tile_width: int = 128, tile_height: int = 128,
                                subpatch_size: int = 8, observer_elevation_m: float = 0.0,
                                device_out: int, degrees: bool = False,
                                pass_seconds: np.ndarray | None = None) -> None:
        """Device-resident march: segment and output device pointers (ints)."""
        handles = (ctypes.c_void_p * len(dems))(*[d.handle.value for d in dems])
        call("ls200_march_all_passes_device", self._ctx, ctypes.c_void_p(device_segments),
             int(azimuth_count), int(center_count), len(dems), handles, int(tile_column),
             int(tile_row), int(tile_width), int(tile_height), int(subpatch_size),
             float(observer_elevation_m), ctypes.c_void_p(device_out), 1 if degrees else 0,
             None if pass_seconds is None else pass_seconds.ctypes.data)

    def generate_segments_device(self, dems, device_segments: int, *, tile_column: int,
                                 tile_row: int, tile_width: int = 128,
                                 azimuth_count: int = 1440,
                                 maximum_distance_m: float = 1_000_000.0,
                                 observer_elevation_m: float = 0.0,
                                 subpatch_size: int = 8) -> None:
        """Segments into a device buffer of A*C*D*18 float32 (pointer int)."""
        handles = (ctypes.c_void_p * len(dems))(*[d.handle.value for d in dems])
        call("ls200_segments_device", self._ctx, handles, len(dems), int(tile_column),
             int(tile_row), int(tile_width), int(azimuth_count), float(maximum_distance_m),
             float(observer_elevation_m), int(subpatch_size), ctypes.c_void_p(device_segments))

    def march_sites(self, tiles, *, device_out: int, azimuth_count: int = 1440,
                    subpatch_size: int = 8, traversal: str = "ladder",
                    degrees: bool = False) -> tuple[float, float]:
        """Every tile of a multi-site batch in one persistent launch into
        ``device_out`` (tile_count x 16384 x azimuth_count float32, pixel-major
        per tile).  Returns (segment + setup seconds, march seconds)."""
        if traversal not in TRAVERSALS:
            raise ValueError(f"traversal must be one of {sorted(TRAVERSALS)}")
        structs, _keep = site_tile_structs(tiles)
        seconds = np.zeros(2, dtype=np.float64)
        call("ls200_march_sites", self._ctx, ctypes.cast(structs, ctypes.c_void_p), len(structs),
             int(azimuth_count),
             int(subpatch_size), TRAVERSALS[traversal], 1 if degrees else 0,
             ctypes.c_void_p(device_out), seconds.ctypes.data)
        return float(seconds[0]), float(seconds[1])

    def set_batch_config(self, config: BatchConfig) -> None:
        """Launch configuration of :meth:`march_sites` (results do not depend on it)."""
        call("ls200_set_batch_config", self._ctx, int(config.lanes_per_azimuth),
             int(config.min_blocks))

    def batch_config(self) -> BatchConfig:
        values = [ctypes.c_int() for _ in range(2)]
        call("ls200_get_batch_config", self._ctx, *[ctypes.byref(v) for v in values])
        return BatchConfig(*(v.value for v in values))

    def check_arithmetic(self) -> tuple[int, int]:
        """(mismatches, checked): results of the march's Newton reciprocal
        that differ in any bit from the IEEE reciprocal, over every pattern
        with |x| >= 2^-64 and both signs; mismatches must be 0."""
        mismatches, checked = ctypes.c_int64(), ctypes.c_int64()
        call("ls200_check_arithmetic", self._ctx, ctypes.byref(mismatches),
             ctypes.byref(checked))
        return int(mismatches.value), int(checked.value)

    def fp32_probe(self, iterations: int = 4096) -> float:
        """Measured FP32 FMA throughput of this device in TFLOP/s."""
        value = ctypes.c_double()
        call("ls200_fp32_probe", self._ctx, int(iterations), ctypes.byref(value))
        return float(value.value)

    def slopes_to_degrees(self, slopes: np.ndarray) -> np.ndarray:
        slopes = np.ascontiguousarray(slopes, dtype=np.float32)
        out = np.empty_like(slopes)
        call("ls200_slopes_to_degrees", self._ctx, slopes.reshape(-1), slopes.size,
             out.reshape(-1))
        return out
