"""``generate_horizons``: the public horizon-tile generator on the B200
(drop-in for src/lunarscout/horizon.py:241-440).

Same signature, validation order, error codes, progress stages, file layout,
resume and cancellation semantics as the reference.  Per patch the whole
chain runs on the device in one C call (``ls200_horizon_tile``): segment
fitting, every DEM pass of the hierarchical march, slope -> degrees, edge
padding and, for ``.cbin``, the encoder; only the payload crosses PCIe.  A
writer thread publishes each file (staged write + fsync + rename) while the
next patch computes.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import sys
import time
from collections.abc import Callable, Sequence
from datetime import datetime, timedelta
from numbers import Real
from pathlib import Path
from typing import Any

import numpy as np

from ._native import CudaBackendError, call, pinned_empty
from .contract import AZIMUTH_COUNT, PATCH_SIZE, PIXEL_COUNT, DemGrid
from .errors import (
    CudaError,
    HorizonGenerationError,
    InputError,
    OperationCancelledError,
    is_cuda_runtime_failure,
)
from .file_format import MAX_PAYLOAD_BYTES, RAW_FILE_BYTES, HorizonTileStore
from .pipeline import HorizonPipelineCancelled, enumerate_patches, run_bounded_pipeline
from .progress import ProgressEvent

ProgressCallback = Callable[[float], None]
ProgressEventCallback = Callable[[ProgressEvent], None]
CancellationCheck = Callable[[], bool]

PUBLIC_MAXIMUM_DISTANCE_M = 1_000_000.0
SUBPATCH_SIZE = 8


class HorizonTileGenerator:
    """Device-resident DEM stack producing one encoded tile per call.

    Payloads land in a ring of page-locked buffers; a returned memoryview is
    valid until ``ring`` further tiles have been computed, which the bounded
    pipeline guarantees by its queue capacity (capacity + 2 buffers).
    """

    def __init__(self, dems: Sequence[DemGrid], *, pyramids=None, device_id: int = 0,
                 session=None, ring: int = 3) -> None:
        from .cuda_backend import CudaSession

        if not dems:
            raise ValueError("at least one DEM is required")
        self._own_session = session is None
        self.session = CudaSession(device_id) if session is None else session
        try:
            if pyramids is None:
                pyramids = [self.session.build_max_pyramid(dem) for dem in dems]
            self.pyramids = tuple(pyramids)
            self.device_dems = [self.session.upload_pyramid(p, dem)
                                for p, dem in zip(self.pyramids, dems)]
        except BaseException:
            self.close()
            raise
        self.primary = dems[0]
        self._handles = (ctypes.c_void_p * len(self.device_dems))(
            *[dem.handle.value for dem in self.device_dems])
        self._ring = max(int(ring), 1)
        self._buffers: dict[bool, list[np.ndarray]] = {True: [], False: []}
        self._next = {True: 0, False: 0}

    def close(self) -> None:
        for dem in getattr(self, "device_dems", []):
            dem.close()
        self.device_dems = []
        if self._own_session and getattr(self, "session", None) is not None:
            self.session.close()
            self.session = None

    def __enter__(self) -> "HorizonTileGenerator":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def _buffer(self, compress: bool) -> np.ndarray:
        buffers = self._buffers[compress]
        index = self._next[compress]
        self._next[compress] = (index + 1) % self._ring
        if index >= len(buffers):
            buffers.append(pinned_empty(MAX_PAYLOAD_BYTES if compress else RAW_FILE_BYTES,
                                        np.uint8))
        return buffers[index]

    def compute(self, tile_x: int, tile_y: int, *, observer_elevation_m: float = 0.0,
                compress: bool = True,
                maximum_distance_m: float = PUBLIC_MAXIMUM_DISTANCE_M) -> memoryview:
        """The file payload of one tile (.cbin bytes or little-endian .bin)."""
        buffer = self._buffer(compress)
        size = ctypes.c_int64()
        call("ls200_horizon_tile", self.session.context, self._handles, len(self.device_dems),
             int(tile_x), int(tile_y), AZIMUTH_COUNT, float(maximum_distance_m),
             float(observer_elevation_m), SUBPATCH_SIZE, 1 if compress else 0,
             buffer.ctypes.data, buffer.size, ctypes.byref(size))
        return memoryview(buffer)[: size.value]

    def degrees(self, tile_x: int, tile_y: int, *, observer_elevation_m: float = 0.0,
                maximum_distance_m: float = PUBLIC_MAXIMUM_DISTANCE_M) -> np.ndarray:
        """float32[16384, 1440] degrees of one tile (a copy)."""
        payload = self.compute(tile_x, tile_y, observer_elevation_m=observer_elevation_m,
                               compress=False, maximum_distance_m=maximum_distance_m)
        return np.frombuffer(payload, dtype="<f4").reshape(PIXEL_COUNT, AZIMUTH_COUNT).copy()


class BatchedTileGenerator:
    """Payloads of many patches from one persistent march per batch
    (``CudaSession.march_sites``): on the first request for a patch it
    marches that patch and the next ``batch_tiles - 1`` pending patches
    together, pads and encodes each on the device and keeps the payloads
    until they are asked for.  ``traversal="exact"`` gives the per-tile
    path's bytes; ``"ladder"`` the skip-ladder traversal (same distance from
    the FP64 restatement, several times faster on long rays)."""

    def __init__(self, dems: Sequence[DemGrid], patches, *, session, pyramids=None,
                 batch_tiles: int = 16, traversal: str = "exact",
                 observer_elevation_m: float = 0.0,
                 maximum_distance_m: float = PUBLIC_MAXIMUM_DISTANCE_M,
                 is_done: Callable | None = None) -> None:
        import torch

        from .cuda_backend import SiteTile
        from .file_format import TileCodec

        if batch_tiles < 1:
            raise ValueError("batch_tiles must be positive")
        self.session = session
        if pyramids is None:
            pyramids = [session.build_max_pyramid(dem) for dem in dems]
        self.device_dems = [session.upload_pyramid(p, dem) for p, dem in zip(pyramids, dems)]
        self.primary = dems[0]
        self.patches = list(patches)
        self.position = {(p.tile_x, p.tile_y): i for i, p in enumerate(self.patches)}
        self.batch_tiles = int(batch_tiles)
        self.traversal = traversal
        self.observer = float(observer_elevation_m)
        self.distance = float(maximum_distance_m)
        self.is_done = is_done or (lambda patch: False)
        self.codec = TileCodec(context=session.context)
        self._site_tile = SiteTile
        self.degrees = torch.empty((self.batch_tiles, PIXEL_COUNT * AZIMUTH_COUNT),
                                   dtype=torch.float32, device="cuda")
        self.payload = torch.empty(MAX_PAYLOAD_BYTES, dtype=torch.uint8, device="cuda")
        self.ready: dict = {}

    def close(self) -> None:
        for dem in self.device_dems:
            dem.close()
        self.device_dems = []
        self.ready.clear()

    def _march(self, batch, compress: bool) -> None:
        import torch

        tiles = [self._site_tile(tuple(self.device_dems), p.tile_x, p.tile_y, self.distance,
                                 self.observer) for p in batch]
        torch.cuda.synchronize()
        self.session.march_sites(tiles, device_out=self.degrees.data_ptr(),
                                 azimuth_count=AZIMUTH_COUNT, traversal=self.traversal,
                                 degrees=True)
        for i, patch in enumerate(batch):
            grid = self.degrees[i].view(PATCH_SIZE, PATCH_SIZE, AZIMUTH_COUNT)
            if patch.width < PATCH_SIZE:
                grid[:, patch.width:] = -50.0
            if patch.height < PATCH_SIZE:
                grid[patch.height:] = -50.0
            torch.cuda.synchronize()
            if compress:
                size = self.codec.encode_device(self.degrees[i].data_ptr(),
                                                self.payload.data_ptr())
                data = self.payload[:size].cpu().numpy().tobytes()
            else:
                data = self.degrees[i].cpu().numpy().astype("<f4", copy=False).tobytes()
            self.ready[(patch.tile_x, patch.tile_y)] = data

    def compute(self, patch, *, compress: bool = True) -> bytes:
        key = (patch.tile_x, patch.tile_y)
        if key not in self.ready:
            batch = [patch]
            for candidate in self.patches[self.position[key] + 1:]:
                if len(batch) == self.batch_tiles:
                    break
                if (candidate.tile_x, candidate.tile_y) not in self.ready and \
                        not self.is_done(candidate):
                    batch.append(candidate)
            self._march(batch, compress)
        return self.ready.pop(key)


class _HorizonProgressAdapter:
    """Private pipeline events -> public ProgressEvent / fraction callbacks
    (ls/horizon.py:43-134): prepare 0.10, patches 0.15 + 0.85 * done/total,
    complete 1.0, fractions never decrease."""

    def __init__(self, output_directory: Path, *, verbose: bool,
                 progress_callback: ProgressCallback | None,
                 progress_event_callback: ProgressEventCallback | None) -> None:
        self.output_directory = output_directory
        self.verbose = verbose
        self.progress_callback = progress_callback
        self.progress_event_callback = progress_event_callback
        self._last_fraction: float | None = None
        self._started: float | None = None
        self.callback_error: BaseException | None = None

    def _timing(self, event: ProgressEvent) -> str:
        if event.stage == "process_patches" and self._started is None:
            self._started = time.monotonic()
        if self._started is None or event.completed <= 0:
            return "    --.-- s/patch | ETA -------------------"
        per_patch = (time.monotonic() - self._started) / event.completed
        eta = datetime.now().astimezone() + timedelta(
            seconds=per_patch * max(0, event.total - event.completed))
        return f"{per_patch:8.2f} s/patch | ETA {eta:%Y-%m-%d %H:%M:%S}"

    def __call__(self, private: Any) -> None:
        stage = str(private.stage)
        completed, total = int(private.processed_patches), int(private.total_patches)
        if stage == "prepare_patches":
            fraction = 0.1
        elif stage == "process_patches":
            fraction = 0.15 + 0.85 * (0.0 if total == 0 else completed / total)
        elif stage == "complete":
            fraction = 1.0
        else:
            fraction = min(1.0, max(0.0, float(private.percent) / 100.0))
        if self._last_fraction is not None:
            fraction = max(self._last_fraction, fraction)
        tile_y = tile_x = None
        if private.file_name:
            parts = str(private.file_name).split("_")
            if len(parts) >= 3:
                try:
                    tile_y, tile_x = int(parts[1]), int(parts[2])
                except ValueError:
                    pass
        event = ProgressEvent("horizons", stage, completed, total, fraction, "cuda",
                              str(private.message), tile_y, tile_x, self.output_directory)
        if self.verbose:
            if stage == "prepare_patches":
                print("horizons: using cuda backend", file=sys.stdout, flush=True)
            print(f"horizons: {stage:<16} {completed:6d}/{total:<6d} | {self._timing(event)}",
                  file=sys.stdout, flush=True)
        if self.progress_event_callback is not None:
            try:
                self.progress_event_callback(event)
            except BaseException as error:
                self.callback_error = error
                raise
        if self.progress_callback is not None and fraction != self._last_fraction:
            try:
                self.progress_callback(fraction)
            except BaseException as error:
                self.callback_error = error
                raise
            self._last_fraction = fraction


def _load_pyramids(session, dems, dem_paths):
    """Sibling .pyr.bin caches; a missing or invalid one is rebuilt on the
    device and atomically replaced (ls/horizon.py:168-177)."""
    from .dem_io import load_max_pyramid_cache, pyramid_cache_path, write_max_pyramid_cache

    pyramids = []
    for dem, path in zip(dems, dem_paths, strict=True):
        cache = pyramid_cache_path(path)
        try:
            pyramid = load_max_pyramid_cache(dem, cache)
        except (OSError, ValueError):
            pyramid = session.build_max_pyramid(dem)
            write_max_pyramid_cache(pyramid, cache)
        pyramids.append(pyramid)
    return tuple(pyramids)


def run_horizon_pipeline(dems: Sequence[DemGrid], output_directory, *,
                         observer_height_m: float = 0.0, compress: bool = True,
                         overwrite: bool = False, dem_paths: Sequence[Path] | None = None,
                         maximum_distance_m: float = PUBLIC_MAXIMUM_DISTANCE_M,
                         device_id: int = 0, progress_callback=None,
                         cancellation_requested: CancellationCheck | None = None,
                         batch_tiles: int = 0, traversal: str = "exact"):
    """Tiles of every pending patch of ``dems[0]`` into ``output_directory``
    (the private pipeline behind the facade; raises the pipeline's own errors).
    ``batch_tiles`` > 0 marches that many patches per persistent launch."""
    from .cuda_backend import CudaSession

    output = Path(output_directory)
    primary = dems[0]
    store = HorizonTileStore(output)
    writer_queue_capacity = 1
    patches = enumerate_patches(primary.width, primary.height)
    session = CudaSession(device_id)
    try:
        pyramids = (_load_pyramids(session, dems, dem_paths) if dem_paths is not None
                    else None)
        if batch_tiles > 0:
            generator = BatchedTileGenerator(
                dems, patches, session=session, pyramids=pyramids, batch_tiles=batch_tiles,
                traversal=traversal, observer_elevation_m=observer_height_m,
                maximum_distance_m=maximum_distance_m,
                is_done=lambda p: not overwrite and store.find_existing_path(
                    p.tile_y, p.tile_x, observer_height_m) is not None)
        else:
            if traversal != "exact":
                raise ValueError("the per-tile path marches the reference traversal only")
            generator = HorizonTileGenerator(dems, pyramids=pyramids, session=session,
                                             ring=writer_queue_capacity + 2)
        try:
            def compute(patch):
                if batch_tiles > 0:
                    return generator.compute(patch, compress=compress)
                return generator.compute(patch.tile_x, patch.tile_y,
                                         observer_elevation_m=observer_height_m,
                                         compress=compress,
                                         maximum_distance_m=maximum_distance_m)

            def write(patch, payload):
                return store.write_payload(patch.tile_y, patch.tile_x, observer_height_m,
                                           payload, compress=compress)

            return run_bounded_pipeline(
                patches,
                store=store, compute_patch=compute, write_patch=write,
                observer_elevation_m=observer_height_m, skip_existing=not overwrite,
                writer_queue_capacity=writer_queue_capacity,
                progress_callback=progress_callback,
                cancellation_requested=cancellation_requested)
        finally:
            generator.close()
    finally:
        session.close()


def _validate(output_directory, observer_height_m, compress, overwrite, verbose,
              progress_callback, progress_event_callback, cancellation_requested) -> Path:
    output = Path(output_directory).expanduser().resolve()
    if output.exists() and not output.is_dir():
        raise InputError("Horizon output must be a directory path.",
                         code="horizon_output_is_file", details={"path": str(output)})
    if (isinstance(observer_height_m, bool) or not isinstance(observer_height_m, Real)
            or not np.isfinite(observer_height_m)
            or not 0.0 <= float(observer_height_m) < 100.0):
        raise InputError(
            "observer_height_m must be finite and between 0.0 and 100.0 meters.",
            code="horizon_observer_height_invalid",
            details={"observer_height_m": observer_height_m})
    for name, value in (("compress", compress), ("overwrite", overwrite), ("verbose", verbose)):
        if not isinstance(value, bool):
            raise InputError(f"{name} must be a bool.", code="horizon_option_invalid",
                             details={"argument": name})
    for name, callback in (("progress_callback", progress_callback),
                           ("progress_event_callback", progress_event_callback),
                           ("cancellation_requested", cancellation_requested)):
        if callback is not None and not callable(callback):
            raise InputError(f"{name} must be callable or None.",
                             code="horizon_callback_invalid", details={"argument": name})
    if cancellation_requested is not None and cancellation_requested():
        raise OperationCancelledError("Horizon generation was cancelled.",
                                      code="horizon_generation_cancelled",
                                      details={"path": str(output)})
    return output


def _check_grid(primary: DemGrid) -> None:
    last_x = ((primary.width - 1) // PATCH_SIZE) * PATCH_SIZE
    last_y = ((primary.height - 1) // PATCH_SIZE) * PATCH_SIZE
    if last_x > 99_999 or last_y > 99_999:
        raise InputError("The primary DEM exceeds the horizon filename coordinate range.",
                         code="horizon_grid_too_large",
                         details={"width": primary.width, "height": primary.height})


def _run_mapped(dems, output: Path, adapter: _HorizonProgressAdapter, **options) -> Path:
    """Run the pipeline and map failures to the public errors
    (ls/horizon.py:405-440)."""
    try:
        run_horizon_pipeline(dems, output, progress_callback=adapter, **options)
        return output
    except Exception as error:
        if adapter.callback_error is error:
            raise
        if isinstance(error, HorizonPipelineCancelled):
            raise OperationCancelledError("Horizon generation was cancelled.",
                                          code="horizon_generation_cancelled",
                                          details={"path": str(output)}) from error
        if isinstance(error, CudaBackendError):
            raise CudaError("A compatible NVIDIA CUDA device is required for horizon generation.",
                            code="cuda_horizon_unavailable",
                            details={"error": str(error)}) from error
        if is_cuda_runtime_failure(error):
            raise CudaError("CUDA horizon generation failed during execution.",
                            code="cuda_horizon_execution_failed",
                            details={"error": str(error)}) from error
        raise HorizonGenerationError(
            "Horizon generation failed.",
            code="horizon_storage_failed" if isinstance(error, OSError)
            else "horizon_generation_failed",
            details={"path": str(output), "error": str(error)}) from error


def generate_horizons(
    output_directory: str | Path,
    dem_paths: Sequence[str | Path],
    *,
    observer_height_m: float = 0.0,
    compress: bool = True,
    overwrite: bool = False,
    verbose: bool = False,
    progress_callback: ProgressCallback | None = None,
    progress_event_callback: ProgressEventCallback | None = None,
    cancellation_requested: CancellationCheck | None = None,
) -> Path:
    """Generate 128-pixel horizon tiles (1440 float32 azimuths per pixel,
    0.25 deg spacing, sample 0 north) for the primary DEM ``dem_paths[0]``,
    later DEMs extending the terrain.  Complete existing tiles are skipped
    unless ``overwrite``; each DEM keeps a sibling ``.pyr.bin`` cache.
    Returns the resolved output directory."""
    if isinstance(dem_paths, (str, bytes, Path)):
        raise InputError("dem_paths must be a sequence ordered primary DEM first.",
                         code="horizon_dem_paths_invalid")
    try:
        resolved = tuple(Path(path).expanduser().resolve() for path in dem_paths)
    except (TypeError, ValueError, OSError) as error:
        raise InputError("dem_paths must contain filesystem paths.",
                         code="horizon_dem_paths_invalid") from error
    if not resolved:
        raise InputError("At least one DEM path is required.", code="horizon_dem_paths_empty")
    missing = tuple(str(path) for path in resolved if not path.is_file())
    if missing:
        raise InputError("A horizon DEM path does not identify a file.",
                         code="horizon_dem_not_found", details={"paths": missing})
    output = _validate(output_directory, observer_height_m, compress, overwrite, verbose,
                       progress_callback, progress_event_callback, cancellation_requested)
    from .dem_io import DemFormatError, load_dem

    try:
        dems = tuple(load_dem(path) for path in resolved)
    except DemFormatError as error:
        raise InputError("A horizon DEM cannot be read.", code="horizon_dem_unreadable",
                         details={"error": str(error)}) from error
    _check_grid(dems[0])
    adapter = _HorizonProgressAdapter(output, verbose=verbose,
                                      progress_callback=progress_callback,
                                      progress_event_callback=progress_event_callback)
    return _run_mapped(dems, output, adapter, dem_paths=resolved,
                       observer_height_m=float(observer_height_m), compress=compress,
                       overwrite=overwrite, cancellation_requested=cancellation_requested)


def generate_horizons_from_grids(
    output_directory: str | Path,
    dems: Sequence[DemGrid],
    *,
    observer_height_m: float = 0.0,
    compress: bool = True,
    overwrite: bool = False,
    maximum_distance_m: float = PUBLIC_MAXIMUM_DISTANCE_M,
    verbose: bool = False,
    progress_callback: ProgressCallback | None = None,
    progress_event_callback: ProgressEventCallback | None = None,
    cancellation_requested: CancellationCheck | None = None,
    batch_tiles: int = 0,
    traversal: str = "exact",
) -> Path:
    """``generate_horizons`` for in-memory DEMs (no pyramid cache files);
    ``maximum_distance_m`` is the private ray range of
    build_subpatch_segments_numba (the public path fixes 1,000 km).
    ``batch_tiles`` > 0 marches that many patches per persistent launch;
    ``traversal="ladder"`` (batched only) uses the skip ladder instead of the
    reference traversal (not bit-identical to the reference's tiles);
    ``"relative"`` / ``"relative-ladder"`` (batched only) march those
    traversals in the relative FP32 arithmetic (closer to the FP64
    restatement, not bit-identical to the reference's tiles)."""
    if not dems or not all(isinstance(dem, DemGrid) for dem in dems):
        raise InputError("dems must be a non-empty sequence of DemGrid, primary first.",
                         code="horizon_dem_paths_invalid")
    if isinstance(batch_tiles, bool) or not isinstance(batch_tiles, int) or batch_tiles < 0:
        raise InputError("batch_tiles must be a non-negative integer.",
                         code="horizon_option_invalid", details={"argument": "batch_tiles"})
    if (traversal not in ("exact", "ladder", "relative", "relative-ladder")
            or (traversal != "exact" and batch_tiles == 0)):
        raise InputError("traversal must be 'exact', or 'ladder', 'relative' or "
                         "'relative-ladder' with batch_tiles > 0.",
                         code="horizon_option_invalid", details={"argument": "traversal"})
    if not (isinstance(maximum_distance_m, Real) and np.isfinite(maximum_distance_m)
            and maximum_distance_m > 0.0):
        raise InputError("maximum_distance_m must be finite and positive.",
                         code="horizon_option_invalid",
                         details={"argument": "maximum_distance_m"})
    output = _validate(output_directory, observer_height_m, compress, overwrite, verbose,
                       progress_callback, progress_event_callback, cancellation_requested)
    _check_grid(dems[0])
    adapter = _HorizonProgressAdapter(output, verbose=verbose,
                                      progress_callback=progress_callback,
                                      progress_event_callback=progress_event_callback)
    return _run_mapped(tuple(dems), output, adapter, observer_height_m=float(observer_height_m),
                       compress=compress, overwrite=overwrite,
                       maximum_distance_m=float(maximum_distance_m),
                       cancellation_requested=cancellation_requested,
                       batch_tiles=batch_tiles, traversal=traversal)


__all__ = ["BatchedTileGenerator", "HorizonTileGenerator", "generate_horizons",
           "generate_horizons_from_grids", "run_horizon_pipeline"]
